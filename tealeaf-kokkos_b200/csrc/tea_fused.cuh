// Fused kernels of the whole-solve path (ext_tea_leaf_solve_).
//
// One chunk, every face external.  The reference keeps each halo equal to the
// reflection of the interior whenever a stencil reads it (update_halo after every
// iteration, tealeaf_2d/tea_solve.f90:489, 632, 704), so these kernels read a
// neighbour outside the inner domain from its reflected interior cell instead of
// from the halo: same value, same arithmetic, no halo maintenance inside the loop.
//
// Stencil kernels stream: lanes own columns and march down rows (2D) or planes (3D),
// keeping the stencil operand of three rows/planes in registers and the loads of the next
// ones in flight; where the operand is itself an update (CG's p = beta p + r) it is
// computed as it is loaded.  Buffers that a sweep both reads at neighbours and rewrites
// (p, u, sd) are double-buffered.
//
// Scalar recurrences (alpha = rro/pw, beta = rrn/rro, ...) and the loop test of
// tea_leaf() run in the last block of the reducing kernel, so one iteration is two
// (CG), one (Chebyshev, Jacobi) or 2 + inner-steps (PPCG) launches, captured in a
// CUDA graph whose while-node reads the continue flag set there.
#pragma once

#include <type_traits>
#include "tea_chunk.cuh"


namespace tea {

enum { PHASE_CG = 0, PHASE_CHEBY = 1, PHASE_PPCG = 2, PHASE_JACOBI = 3 };
enum { EXIT_NONE = 0, EXIT_CONVERGED = 1, EXIT_MAXITER = 2, EXIT_PHASE = 3 };
enum { SOLVER_JACOBI = 1, SOLVER_CG = 2, SOLVER_CHEBY = 3, SOLVER_PPCG = 4 };

// Device-resident scalars of one solve (the local variables of tea_leaf()).
struct SolveState {
    double rro, pw, rrn, alpha, beta, error, eps, theta;
    double last_alpha, last_beta, epslim;
    int n;                // the iteration being executed (Fortran DO variable)
    int cont;             // loop continues
    int exit_reason;
    int pending_p;        // p = last_beta p + (z|r) still to apply
    int pending_u;        // u += last_alpha p still to apply
    int par_u, par_p;     // which buffer of u / p is current
    int cheby_calc_steps;
    int est_itc;
    int resid_pending;    // Jacobi: residual check due this iteration
    int solver, precond, max_iters, presteps, errswitch, inner_steps;
    int nonfinite;
    // FP32 inner solve of the defect-correction form.
    int n_inner, inner_max;
    int inner_cheby;     // the inner solve: 0 CG, 1 Chebyshev, 2 PPCG
    int inner_diverged;  // the inner Chebyshev residual stalled or grew (bounds too narrow)
    double cheby_rho2;   // squared Chebyshev contraction per iteration for the bounds in use
    double tol2;
    // The first inner CG of a Chebyshev or PPCG deck also stops at the plain solve's switch
    // test (sum r^2 <= switch_err after switch_min iterations); 0 when it does not apply.
    double switch_err;
    int switch_min;
};

struct FusedArgs {
    Geom g;
    double* u[2];
    double* p[2];
    double* sd[2];
    double *r, *w, *z, *mi, *u0, *kx, *ky, *kz;
    double *cg_alphas, *cg_betas;          // [max_iters + 2], indexed by n
    const double *ch_alphas, *ch_betas;    // Chebyshev / PPCG coefficients
    SolveState* st;
    RedScratch red;
    cudaGraphConditionalHandle handle;
    int use_handle;
    int tiles_x, tiles_y, zseg;
    long ntiles;
    int step;    // PPCG inner step (1-based) of this launch
    int seg_rows;  // rows per warp segment of the 2D ring kernels (set per launch)
    int timing;  // measurement launches: the last block leaves the solve state untouched
    int r_in_w;  // PPCG: sweep B leaves r in the w array and the two-step passes start there
    // FP32 arrays of the defect-correction form (same pitched layout, float elements).
    float *kx32, *ky32, *kz32, *r32, *w32, *d32;
    float* p32[2];
    float* dc32[2];  // iterate of the inner Chebyshev solve (ping-pong over d32, w32)
    float* sd32[2];  // sd of the inner PPCG solve
};


// Reflection of a padded index into the inner domain (depth 1 and 2): HALO_PAD-1-f
// maps to HALO_PAD+f and N-HALO_PAD+f to N-HALO_PAD-1-f, as UpdateHalo copies them.
__device__ __forceinline__ int refl(int k, int n)
{
    return k < HALO_PAD ? 2 * HALO_PAD - 1 - k : (k >= n - HALO_PAD ? 2 * (n - HALO_PAD) - 1 - k : k);
}

template <class T>
struct NbT {
    T c, xm, xp, ym, yp, zm, zp;
};
using Nb = NbT<double>;

// SMVP with the operand taken from staged neighbours (same expression as smvp()).
__device__ __forceinline__ double smvp_nb(const Nb& a, const double* __restrict__ kx,
                                          const double* __restrict__ ky, const double* __restrict__ kz,
                                          long i, long pitch, long page)
{
    const double kx0 = kx[i], kx1 = kx[i + 1], ky0 = ky[i], ky1 = ky[i + pitch];
#if TEA_DIM == 2
    (void)kz;
    (void)page;
    return (1.0 + (kx1 + kx0) + (ky1 + ky0)) * a.c - (kx1 * a.xp + kx0 * a.xm) - (ky1 * a.yp + ky0 * a.ym);
#else
    const double kz0 = kz[i], kz1 = kz[i + page];
    return (1.0 + (kx1 + kx0) + (ky1 + ky0) + (kz1 + kz0)) * a.c - (kx1 * a.xp + kx0 * a.xm)
        - (ky1 * a.yp + ky0 * a.ym) - (kz1 * a.zp + kz0 * a.zm);
#endif
}

// The operator and the Jacobi update from staged neighbours and register-held
// coefficients (kx0 = Kx[i], kx1 = Kx[i+1], ky1 = Ky[i+pitch], kz1 = Kz[i+page]); the
// same expressions, in the same order, as smvp() and JacobiSolve.
template <class T>
__device__ __forceinline__ T smvp_k(const NbT<T>& a, T kx0, T kx1, T ky0, T ky1, T kz0, T kz1)
{
    const T one = (T)1;
#if TEA_DIM == 2
    (void)kz0;
    (void)kz1;
    return (one + (kx1 + kx0) + (ky1 + ky0)) * a.c - (kx1 * a.xp + kx0 * a.xm) - (ky1 * a.yp + ky0 * a.ym);
#else
    return (one + (kx1 + kx0) + (ky1 + ky0) + (kz1 + kz0)) * a.c - (kx1 * a.xp + kx0 * a.xm)
        - (ky1 * a.yp + ky0 * a.ym) - (kz1 * a.zp + kz0 * a.zm);
#endif
}

__device__ __forceinline__ double jacobi_k(double u0, const Nb& a, double kx0, double kx1, double ky0, double ky1,
                                           double kz0, double kz1)
{
#if TEA_DIM == 2
    (void)kz0;
    (void)kz1;
    return (u0 + (kx1 * a.xp + kx0 * a.xm) + (ky1 * a.yp + ky0 * a.ym)) / (1.0 + (kx0 + kx1) + (ky0 + ky1));
#else
    return (u0 + (kx1 * a.xp + kx0 * a.xm) + (ky1 * a.yp + ky0 * a.ym) + (kz1 * a.zp + kz0 * a.zm))
        / (1.0 + (kx0 + kx1) + (ky0 + ky1) + (kz0 + kz1));
#endif
}

// ------------------------------------------------------------------ loop control

__device__ __forceinline__ bool switch_check(const SolveState& s, int n)
{
    // tealeaf_2d/tea_solve.f90:173-179
    if (s.errswitch) return (s.cheby_calc_steps > 0) || ((s.error <= s.epslim) && (n >= 20));
    return (n >= s.presteps) && (s.error <= 1.0);
}

// End of iteration s.n: the EXIT test of tealeaf_2d/tea_solve.f90:501, the DO bound, and
// whether the next iteration still belongs to this loop's branch.  On exit s.n is the
// Fortran n after the loop (the printed count is n-1); otherwise it advances.
__device__ void end_iteration(const FusedArgs& a, SolveState& s, int phase)
{
    const int n = s.n;
    int cont = 1, reason = EXIT_NONE;
    if (fabs(s.error) < s.eps) {
        cont = 0;
        reason = EXIT_CONVERGED;
    } else if (n + 1 > s.max_iters) {
        cont = 0;
        reason = EXIT_MAXITER;
    } else if (s.solver == SOLVER_CHEBY || s.solver == SOLVER_PPCG) {
        const bool sw = switch_check(s, n + 1);
        if ((phase == PHASE_CG) == sw) {
            cont = 0;
            reason = EXIT_PHASE;
        }
    }
    if (reason != EXIT_CONVERGED) s.n = n + 1;
    s.cont = cont;
    s.exit_reason = reason;
    if (a.use_handle) cudaGraphSetConditional(a.handle, cont ? 1u : 0u);
}

// ------------------------------------------------------------------ generic stencil drivers

// Op interface (one Op per fused stencil sweep):
//   using T (operand and coefficient type); static constexpr int NV (reduced values);
//   static constexpr bool kReduce;
//   skip(a)            -- the whole launch is a no-op (uniform)
//   begin(a)           -- read the solve state into registers
//   coef_x/y/z(a)      -- coefficient arrays
//   Raw load_raw(a, i) / T stage_raw(Raw)  -- loads behind the stencil operand at cell i,
//                                           and the operand computed from them
//   In load_in(a, i)   -- the other per-cell inputs of the interior update
//   interior_k(a, i, nb, raw_c, in, kx0, kx1, ky0, ky1, kz0, kz1, acc)
//   control(a, v)      -- last block, lane 0, with the rounded sums v[0..NV)

constexpr int SW = 4;      // warps per block (2D)
constexpr int SY = 32;     // rows per column segment (2D)
constexpr int SBLOCK = 32 * SW;

// 2D register streaming with one row of software prefetch: the loads of row j+2 are in
// flight while row j is computed.  Per row each lane carries the raw inputs of the
// operand (Op::Raw) and the interior inputs (Op::In plus Kx, Ky); Kx of the right face
// comes from the next lane, Ky of the upper face from the next row's bundle.  Inactive
// lanes past the last column shadow it for the operand and load the boundary face's Kx,
// so the last active lane sees the reflection and the stored boundary coefficient.
template <class Op>
__global__ void __launch_bounds__(SBLOCK) k_pipe2d(FusedArgs a)
{
    using Raw = typename Op::Raw;
    using In = typename Op::In;
    using T = typename Op::T;
    constexpr int NV = Op::NV;
    struct Bundle {
        In in;
        T kx, kxe;
    };
    Op op;
    if (op.skip(a)) return;
    op.begin(a);
    const Geom& g = a.g;
    const T* __restrict__ KX = op.coef_x(a);
    const T* __restrict__ KY = op.coef_y(a);
    DDVec<NV> acc;
    acc.zero();
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int xlast = g.X - HALO_PAD - 1;
    const int ylast = g.Y - HALO_PAD - 1;
    for (long t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
        const int tx = (int)(t % a.tiles_x), ty = (int)(t / a.tiles_x);
        const int wx = HALO_PAD + tx * SBLOCK + warp * 32;
        if (wx > xlast) continue;  // the whole warp is past the last column
        const int kk = wx + lane;
        const bool active = kk <= xlast;
        const int kc = min(kk, xlast);          // operand column (shadows the last one)
        const int kq = min(kk, xlast + 1);      // coefficient column
        const bool edge = lane == 0 || lane == 31;
        const int ke = lane == 0 ? refl(kc - 1, g.X) : refl(min(kc + 1, xlast + 1), g.X);
        const int j0 = HALO_PAD + ty * SY;
        const int j1 = min(j0 + SY, ylast + 1);
        auto bundle = [&](int jj) {
            Bundle b;
            b.in = op.load_in(a, fidx(g, kc, jj, 0));
            b.kx = KX[fidx(g, kq, jj, 0)];
            b.kxe = lane == 31 ? KX[fidx(g, min(kk + 1, xlast + 1), jj, 0)] : (T)0;
            return b;
        };
        // Pipelines: operand raw inputs two rows ahead, interior bundle one row ahead,
        // Ky two rows ahead (row j+1's Ky is row j's upper-face coefficient).
        Raw rc = op.load_raw(a, fidx(g, kc, j0, 0));
        Raw rp = op.load_raw(a, fidx(g, kc, refl(j0 + 1, g.Y), 0));
        T sm = op.stage_raw(op.load_raw(a, fidx(g, kc, refl(j0 - 1, g.Y), 0)));
        T sc = op.stage_raw(rc);
        Bundle bc = bundle(j0);
        T ky0 = KY[fidx(g, kc, j0, 0)];
        T ky1 = KY[fidx(g, kc, j0 + 1, 0)];
        Raw rec;
        if (edge) rec = op.load_raw(a, fidx(g, ke, j0, 0));
        for (int jj = j0; jj < j1; ++jj) {
            const int jn = min(jj + 1, ylast);
            const Raw rpp = op.load_raw(a, fidx(g, kc, refl(min(jj + 2, ylast + 2), g.Y), 0));
            const Bundle bn = bundle(jn);
            const T ky2 = KY[fidx(g, kc, min(jj + 2, ylast + 1), 0)];
            Raw ren;
            if (edge) ren = op.load_raw(a, fidx(g, ke, jn, 0));
            const T sp = op.stage_raw(rp);
            const T e = edge ? op.stage_raw(rec) : (T)0;
            const T up = __shfl_up_sync(0xffffffffu, sc, 1);
            const T dn = __shfl_down_sync(0xffffffffu, sc, 1);
            const T kxr = __shfl_down_sync(0xffffffffu, bc.kx, 1);
            if (active) {
                NbT<T> nb;
                nb.c = sc;
                nb.xm = lane == 0 ? e : up;
                nb.xp = lane == 31 ? e : dn;
                nb.ym = sm;
                nb.yp = sp;
                nb.zm = nb.zp = (T)0;
                const T kx1 = lane == 31 ? bc.kxe : kxr;
                op.interior_k(a, fidx(g, kk, jj, 0), nb, rc, bc.in, bc.kx, kx1, ky0, ky1, (T)0, (T)0, acc);
            }
            sm = sc;
            sc = sp;
            rc = rp;
            rp = rpp;
            bc = bn;
            ky0 = ky1;
            ky1 = ky2;
            if (edge) rec = ren;
        }
    }
    if (Op::kReduce) grid_reduce_then<NV>(acc, a.red, [&](const double* v) { op.control(a, v); });
}

// 3D register streaming: a block of TY3 + 2 warps covers 32 columns x TY3 rows of one
// x-y tile and marches through a z segment.  Warp w (1..TY3) owns row y0 + w - 1; warps 0
// and TY3 + 1 only stage the operand of the rows just outside the tile.  Each lane keeps
// the operand of planes ii-1, ii, ii+1 of its column in registers (z-neighbours) and the
// raw inputs and interior bundle of the next planes in flight; x-neighbours come by
// shuffle (edge lanes stage their outside neighbour), y-neighbours through a shared plane
// that is double-buffered, so one barrier per plane suffices.
constexpr int TY3 = 8;
constexpr int P3BLOCK = 32 * (TY3 + 2);

template <class Op>
__global__ void __launch_bounds__(P3BLOCK, 2) k_pipe3d(FusedArgs a)
{
    using Raw = typename Op::Raw;
    using In = typename Op::In;
    using T = typename Op::T;
    constexpr int NV = Op::NV;
    struct Bundle {
        In in;
        T kx, ky, ky1, kxe;
    };
    __shared__ T s_pl[2][TY3 + 2][32];
    Op op;
    if (op.skip(a)) return;
    op.begin(a);
    const Geom& g = a.g;
    const T* __restrict__ KX = op.coef_x(a);
    const T* __restrict__ KY = op.coef_y(a);
    const T* __restrict__ KZ = op.coef_z(a);
    DDVec<NV> acc;
    acc.zero();
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const bool owner = warp >= 1 && warp <= TY3;
    const int xlast = g.X - HALO_PAD - 1;
    const int ylast = g.Y - HALO_PAD - 1;
    const int zlast = g.Z - HALO_PAD - 1;
    const long txy = (long)a.tiles_x * a.tiles_y;
    for (long t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
        const int zs = (int)(t / txy);
        const long rxy = t % txy;
        const int tx = (int)(rxy % a.tiles_x), ty = (int)(rxy / a.tiles_x);
        const int kk = HALO_PAD + tx * 32 + lane;
        const bool colok = kk <= xlast;
        const int kc = min(kk, xlast);
        const int kq = min(kk, xlast + 1);
        const bool edge = lane == 0 || lane == 31;
        const int ke = lane == 0 ? refl(kc - 1, g.X) : refl(min(kc + 1, xlast + 1), g.X);
        const int y0 = HALO_PAD + ty * TY3;
        const int jraw = y0 + warp - 1;                      // row of this warp (halo warps outside)
        const bool rowok = owner && jraw <= ylast;
        const int jc = refl(min(jraw, ylast + 1), g.Y);      // operand row (reflected, clamped)
        const int jq = min(max(jraw, HALO_PAD), ylast);      // interior row for loads (valid)
        const bool active = colok && rowok;
        const int z0 = HALO_PAD + zs * a.zseg;
        const int z1 = min(z0 + a.zseg, zlast + 1);
        auto raw_at = [&](int col, int plane) { return op.load_raw(a, fidx(g, col, jc, refl(plane, g.Z))); };
        auto bundle = [&](int plane) {
            Bundle b;
            b.in = op.load_in(a, fidx(g, kc, jq, plane));
            b.kx = KX[fidx(g, kq, jq, plane)];
            b.ky = KY[fidx(g, kc, jq, plane)];
            b.ky1 = KY[fidx(g, kc, jq + 1, plane)];
            b.kxe = lane == 31 ? KX[fidx(g, min(kk + 1, xlast + 1), jq, plane)] : (T)0;
            return b;
        };
        // Pipelines: operand raw inputs two planes ahead, interior bundle one plane ahead,
        // Kz two planes ahead (plane ii+1's Kz is plane ii's upper-face coefficient).
        Raw rc = raw_at(kc, z0);
        Raw rp = raw_at(kc, z0 + 1);
        T sm = op.stage_raw(raw_at(kc, z0 - 1));
        T sc = op.stage_raw(rc);
        Bundle bc;
        T kz0 = 0, kz1 = 0;
        if (owner) {
            bc = bundle(z0);
            kz0 = KZ[fidx(g, kc, jq, z0)];
            kz1 = KZ[fidx(g, kc, jq, z0 + 1)];
        }
        Raw rec;
        if (edge && owner) rec = raw_at(ke, z0);
        int buf = 0;
        for (int ii = z0; ii < z1; ++ii) {
            const int zn = min(ii + 1, zlast);
            const Raw rpp = raw_at(kc, min(ii + 2, zlast + 2));
            Bundle bn;
            T kz2 = 0;
            Raw ren;
            if (owner) {
                bn = bundle(zn);
                kz2 = KZ[fidx(g, kc, jq, min(ii + 2, zlast + 1))];
                if (edge) ren = raw_at(ke, zn);
            }
            const T sp = op.stage_raw(rp);
            s_pl[buf][warp][lane] = sc;
            __syncthreads();
            if (owner) {
                const T e = edge ? op.stage_raw(rec) : (T)0;
                const T up = __shfl_up_sync(0xffffffffu, sc, 1);
                const T dn = __shfl_down_sync(0xffffffffu, sc, 1);
                const T kxr = __shfl_down_sync(0xffffffffu, bc.kx, 1);
                if (active) {
                    NbT<T> nb;
                    nb.c = sc;
                    nb.xm = lane == 0 ? e : up;
                    nb.xp = lane == 31 ? e : dn;
                    nb.ym = s_pl[buf][warp - 1][lane];
                    nb.yp = s_pl[buf][warp + 1][lane];
                    nb.zm = sm;
                    nb.zp = sp;
                    const T kx1 = lane == 31 ? bc.kxe : kxr;
                    op.interior_k(a, fidx(g, kk, jraw, ii), nb, rc, bc.in, bc.kx, kx1, bc.ky, bc.ky1, kz0, kz1,
                                  acc);
                }
                bc = bn;
                kz0 = kz1;
                kz1 = kz2;
                if (edge) rec = ren;
            }
            sm = sc;
            sc = sp;
            rc = rp;
            rp = rpp;
            buf ^= 1;
        }
        __syncthreads();
    }
    if (Op::kReduce) grid_reduce_then<NV>(acc, a.red, [&](const double* v) { op.control(a, v); });
}

// 2D streaming through a per-warp shared-memory ring filled by cp.async.  Each warp owns a
// strip of 32 * VEC columns (VEC adjacent cells per lane: one 16-byte copy, 2 doubles or 4
// floats) and marches down a segment of a.seg_rows rows; the rows of every input array are
// copied asynchronously RP rows ahead of the row being computed, so the data in flight
// lives in shared memory, not in registers.  A ring row also holds the two columns just
// outside the strip (the x-neighbours of its edge cells).  Rows and columns outside the
// inner domain are copied from their reflected interior cell; within the strip the
// right-hand boundary is reflected when the operand is read.  No block barrier: warps are
// independent.
#ifndef TEA_RING_RP
#define TEA_RING_RP 3
#endif
#ifndef TEA_RING_WARPS
#define TEA_RING_WARPS 4
#endif
#ifndef TEA_CHEBY2_RP
#define TEA_CHEBY2_RP 3
#endif
constexpr int RP = TEA_RING_RP;  // rows in flight beyond row j+1
constexpr int RQ = RP + 2;     // ring rows per warp
constexpr int RWARPS = TEA_RING_WARPS;  // warps per block

__device__ __forceinline__ void cp_async_16(void* dst, const void* src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_8(void* dst, const void* src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_4(void* dst, const void* src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

template <class T>
__device__ __forceinline__ void ring_copy_pair(T* dst, const T* src)
{
    if (sizeof(T) == 8) cp_async_16(dst, src);
    else cp_async_8(dst, src);
}
template <class T>
__device__ __forceinline__ void ring_copy_one(T* dst, const T* src)
{
    if (sizeof(T) == 8) cp_async_8(dst, src);
    else cp_async_4(dst, src);
}

// Strip geometry of the 2D ring kernels for element type T: each lane owns VEC adjacent
// cells (one 16-byte copy), a warp a strip of 32 * VEC columns.  A ring row holds the
// strip at offset OFF (16-byte aligned) with the left outside column at OFF - 1 and the
// right one at OFF + STRIP.
template <class T, int V = 16 / (int)sizeof(T)>
struct RingGeom {
    static constexpr int VEC = V;
    static constexpr int STRIP = 32 * VEC;
    static constexpr int OFF = 16 / (int)sizeof(T);  // keeps the strip 16-byte aligned
    static constexpr int WIDTH = STRIP + 2 * OFF;
};

// Cells per lane of a sweep's ring kernel: one 16-byte copy (2 doubles or 4 floats).
template <class Op>
struct RingVec {
    static constexpr int value = 16 / (int)sizeof(typename Op::T);
};
struct OpSweepA32;
struct OpCheby32;
template <class Op>
using RingGeomOf = RingGeom<typename Op::T, RingVec<Op>::value>;

// Sweeps whose ring kernels compute a lane's VEC cells first and then store each output
// array with one vector store (Op::Out, interior_out, store_vec, store_one) instead of one
// scalar store per cell and array.
template <class Op>
struct RingVecStore {
    static constexpr bool value = false;
};
template <>
struct RingVecStore<OpSweepA32> {
    static constexpr bool value = true;
};
template <>
struct RingVecStore<OpCheby32> {
    static constexpr bool value = true;
};

template <class T>
__device__ __forceinline__ void ld_vec(const T* p, T* out);
template <>
__device__ __forceinline__ void ld_vec<double>(const double* p, double* out)
{
    const double2 v = *reinterpret_cast<const double2*>(p);
    out[0] = v.x;
    out[1] = v.y;
}
template <>
__device__ __forceinline__ void ld_vec<float>(const float* p, float* out)
{
    const float4 v = *reinterpret_cast<const float4*>(p);
    out[0] = v.x;
    out[1] = v.y;
    out[2] = v.z;
    out[3] = v.w;
}

// One 16-byte vector store (2 doubles or 4 floats, 16-byte aligned).
template <class T>
__device__ __forceinline__ void st_vec(T* p, const T* v);
template <>
__device__ __forceinline__ void st_vec<double>(double* p, const double* v)
{
    *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]);
}
template <>
__device__ __forceinline__ void st_vec<float>(float* p, const float* v)
{
    *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}

// VEC consecutive elements (8 or 16 bytes, aligned to their size).
template <int VEC, class T>
__device__ __forceinline__ void ld_vecn(const T* p, T* out)
{
    if constexpr (VEC * sizeof(T) == 16) {
        ld_vec(p, out);
    } else {
        static_assert(VEC == 2 && sizeof(T) == 4, "8-byte vectors are float pairs");
        const float2 v = *reinterpret_cast<const float2*>(p);
        out[0] = v.x;
        out[1] = v.y;
    }
}
template <int VEC, class T>
__device__ __forceinline__ void cp_async_vecn(T* dst, const T* src)
{
    if constexpr (VEC * sizeof(T) == 16) cp_async_16(dst, src);
    else cp_async_8(dst, src);
}

template <class Op>
constexpr size_t ring_smem_bytes()
{
    using T = typename Op::T;
    return (size_t)RWARPS * RQ * (Op::NR + Op::NI + 2) * RingGeomOf<Op>::WIDTH * sizeof(T);
}

// The body of k_ring2d after op.begin(), ending with the grid reduction and op.control().
template <class Op>
__device__ __forceinline__ void ring2d_body(const FusedArgs& a, Op& op, unsigned char* s_ring_raw)
{
    using T = typename Op::T;
    constexpr int NV = Op::NV;
    constexpr int NR = Op::NR, NI = Op::NI;
    constexpr int NA = NR + NI + 2;  // + Kx, Ky
    constexpr int AKX = NR + NI, AKY = NR + NI + 1;
    constexpr int VEC = RingGeomOf<Op>::VEC, STRIP = RingGeomOf<Op>::STRIP, OFF = RingGeomOf<Op>::OFF;
    constexpr int RWT = RingGeomOf<Op>::WIDTH;
    const Geom& g = a.g;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    T* ring = reinterpret_cast<T*>(s_ring_raw) + (size_t)warp * RQ * NA * RWT;
    const T* src[NA];
#pragma unroll
    for (int k = 0; k < NR; ++k) src[k] = op.raw_ptr(a, k);
#pragma unroll
    for (int k = 0; k < NI; ++k) src[NR + k] = op.in_ptr(a, k);
    src[AKX] = op.coef_x(a);
    src[AKY] = op.coef_y(a);
    DDVec<NV> acc;
    acc.zero();
    const int xlast = g.X - HALO_PAD - 1;
    const int ylast = g.Y - HALO_PAD - 1;
    const int per_x = (g.nx + STRIP - 1) / STRIP;
    const int per_y = (g.ny + a.seg_rows - 1) / a.seg_rows;
    const long nseg = (long)per_x * per_y;
    const long gw = (long)blockIdx.x * RWARPS + warp, nw = (long)gridDim.x * RWARPS;
    // Last first-column of a lane whose VEC cells stay inside the row (same residue as the
    // lanes' columns modulo VEC, so the copy stays 16-byte aligned); lanes beyond it own
    // no inner cell.
    const int cmax = (int)g.pitch - 2 * VEC + 2;
    for (long sgi = gw; sgi < nseg; sgi += nw) {
        const int xs = (int)(sgi % per_x), ys = (int)(sgi / per_x);
        const int c0 = HALO_PAD + STRIP * xs;
        const int c = c0 + VEC * lane;
        const int cc = min(c, cmax);
        const int j0 = HALO_PAD + a.seg_rows * ys;
        const int j1 = min(j0 + a.seg_rows, ylast + 1);
        const int left = refl(c0 - 1, g.X);
        const int right_op = refl(min(c0 + STRIP, xlast + 1), g.X);
        const int right_k = min(c0 + STRIP, xlast + 1);
        auto slot = [&](int r) { return ring + (size_t)((r - j0 + 1) % RQ) * NA * RWT; };
        // Copy the ring row of grid row r.
        auto issue = [&](int r) {
            if (r <= j1) {
                T* base = slot(r);
                const int srow = refl(min(max(r, 1), ylast + 1), g.Y);
                const int irow = min(max(r, HALO_PAD), ylast + 1);
#pragma unroll
                for (int k = 0; k < NA; ++k) {
                    const T* sp = src[k];
                    if (!sp) continue;
                    const int row = k < NR ? srow : irow;
                    T* d = base + k * RWT;
                    cp_async_vecn<VEC>(d + OFF + VEC * lane, sp + fidx(g, cc, row, 0));
                    if (lane == 0 && k < NR) ring_copy_one(d + OFF - 1, sp + fidx(g, left, row, 0));
                    if (lane == 31 && (k < NR || k == AKX))
                        ring_copy_one(d + OFF + STRIP, sp + fidx(g, k < NR ? right_op : right_k, row, 0));
                }
            }
            cp_async_commit();
        };
        // The operand of ring row r at the lane's cells and at the strip's outside column
        // (left for lane 0, right for lane 31).
        auto stage_row = [&](int r, T* v, T& ve) {
            const T* base = slot(r);
            T x[NR][VEC], xq[NR], xe[NR];
#pragma unroll
            for (int k = 0; k < NR; ++k) {
                ld_vecn<VEC>(base + k * RWT + OFF + VEC * lane, x[k]);
                xe[k] = base[k * RWT + (lane == 0 ? OFF - 1 : OFF + STRIP)];
            }
#pragma unroll
            for (int q = 0; q < VEC; ++q) {
#pragma unroll
                for (int k = 0; k < NR; ++k) xq[k] = x[k][q];
                v[q] = op.stage_raw(op.raw_from(xq));
            }
            ve = op.stage_raw(op.raw_from(xe));
        };
        for (int r = j0 - 1; r <= j0 + RP; ++r) issue(r);
        cp_async_wait<RP>();
        __syncwarp();
        T mv[VEC], cv[VEC], ce;
        stage_row(j0 - 1, mv, ce);  // (the outside column of row j0 - 1 is not needed)
        stage_row(j0, cv, ce);
        for (int jj = j0; jj < j1; ++jj) {
            cp_async_wait<RP - 1>();
            __syncwarp();
            T pv[VEC], pe;
            stage_row(jj + 1, pv, pe);
            const T* cur = slot(jj);
            const T* nxt = slot(jj + 1);
            const T up = __shfl_up_sync(0xffffffffu, cv[VEC - 1], 1);
            const T dn = __shfl_down_sync(0xffffffffu, cv[0], 1);
            T kx[VEC + 1], ky0[VEC], ky1[VEC];
            ld_vecn<VEC>(cur + AKX * RWT + OFF + VEC * lane, kx);
            const T kxn = __shfl_down_sync(0xffffffffu, kx[0], 1);
            kx[VEC] = lane == 31 ? cur[AKX * RWT + OFF + STRIP] : kxn;
            ld_vecn<VEC>(cur + AKY * RWT + OFF + VEC * lane, ky0);
            ld_vecn<VEC>(nxt + AKY * RWT + OFF + VEC * lane, ky1);
            T rv[NR > 0 ? NR : 1][VEC], iv[NI][VEC];
#pragma unroll
            for (int k = 0; k < NR; ++k) ld_vecn<VEC>(cur + k * RWT + OFF + VEC * lane, rv[k]);
#pragma unroll
            for (int k = 0; k < NI; ++k) ld_vecn<VEC>(cur + (NR + k) * RWT + OFF + VEC * lane, iv[k]);
            auto cell_nb = [&](int q) {
                const int cq = c + q;
                NbT<T> nb;
                nb.c = cv[q];
                nb.xm = q == 0 ? (lane == 0 ? ce : up) : cv[q > 0 ? q - 1 : 0];
                nb.xp = cq == xlast ? cv[q] : (q == VEC - 1 ? (lane == 31 ? ce : dn) : cv[q < VEC - 1 ? q + 1 : q]);
                nb.ym = mv[q];
                nb.yp = pv[q];
                nb.zm = nb.zp = (T)0;
                return nb;
            };
            if constexpr (RingVecStore<Op>::value) {
                typename Op::Out o[VEC];
#pragma unroll
                for (int q = 0; q < VEC; ++q) {
                    T rq[NR > 0 ? NR : 1], iq[NI];
#pragma unroll
                    for (int k = 0; k < NR; ++k) rq[k] = rv[k][q];
#pragma unroll
                    for (int k = 0; k < NI; ++k) iq[k] = iv[k][q];
                    o[q] = op.interior_out(cell_nb(q), op.raw_from(rq), op.in_from(iq), kx[q], kx[q + 1], ky0[q], ky1[q],
                                           (T)0, (T)0, acc, c + q <= xlast);
                }
                const long i0 = fidx(g, c, jj, 0);
                if (c + VEC - 1 <= xlast) {
                    op.store_vec(a, i0, o);
                } else {
#pragma unroll
                    for (int q = 0; q < VEC; ++q)
                        if (c + q <= xlast) op.store_one(a, i0 + q, o[q]);
                }
            } else {
#pragma unroll
                for (int q = 0; q < VEC; ++q) {
                    const int cq = c + q;
                    if (cq <= xlast) {
                        T rq[NR > 0 ? NR : 1], iq[NI];
#pragma unroll
                        for (int k = 0; k < NR; ++k) rq[k] = rv[k][q];
#pragma unroll
                        for (int k = 0; k < NI; ++k) iq[k] = iv[k][q];
                        op.interior_k(a, fidx(g, cq, jj, 0), cell_nb(q), op.raw_from(rq), op.in_from(iq), kx[q],
                                      kx[q + 1], ky0[q], ky1[q], (T)0, (T)0, acc);
                    }
                }
            }
#pragma unroll
            for (int q = 0; q < VEC; ++q) {
                mv[q] = cv[q];
                cv[q] = pv[q];
            }
            ce = pe;
            __syncwarp();
            issue(jj + RP + 1);  // into the slot of row jj - 1, which no lane reads any more
        }
        cp_async_wait<0>();
        __syncwarp();
    }
    if (Op::kReduce) grid_reduce_then<NV>(acc, a.red, [&](const double* v) { op.control(a, v); });
}

template <class Op>
__global__ void __launch_bounds__(RWARPS * 32) k_ring2d(FusedArgs a)
{
    extern __shared__ __align__(16) unsigned char s_ring_raw[];
    Op op;
    if (op.skip(a)) return;
    op.begin(a);
    ring2d_body(a, op, s_ring_raw);
}

#if TEA_DIM == 3
// 3D streaming through a block-shared ring of planes filled by cp.async.  A block of TY
// warps owns an x-y tile of 32 * VEC columns by TY rows (warp w: row y0 + w) and marches
// through a segment of a.seg_rows planes.  A ring slot holds one plane of the tile: per
// operand array the tile's rows plus the rows just below and above it, per interior input
// the tile's rows, Kx (with the column right of the strip), Ky (with the row above the
// tile) and Kz; operand rows also carry the two columns just outside the strip.  RP planes
// are in flight beyond plane z+1 (RP + 2 slots).  The operand of planes z-1, z, z+1 at the
// warp's own row stays in registers (z-neighbours), y-neighbours are staged from the slot's
// neighbouring rows (the staging arithmetic is the same, so the values are identical),
// x-neighbours come by shuffle.  One block barrier per plane: after it every warp's copies
// of plane z+1 have landed and no warp still reads the slot that the next copy overwrites.
// Work units (tile, z segment) are ordered segment-major, so tiles that are y-neighbours
// run at the same time and their shared rows are read from L2.  TY and RP are chosen per
// sweep: more resident blocks per SM (short tiles, few slots) hide the per-plane barrier
// better than deeper prefetch does.

// Row offsets of one ring slot.
template <class Op, int TY>
struct Ring3Rows {
    static constexpr int RAW = 0;                               // Op::NR x (TY + 2)
    static constexpr int IN = Op::NR * (TY + 2);                // Op::NI x TY
    static constexpr int KX = IN + Op::NI * TY;                 // TY
    static constexpr int KY = KX + TY;                          // TY + 1
    static constexpr int KZ = KY + TY + 1;                      // TY
    static constexpr int ROWS = KZ + TY;
};

template <class Op, int TY, int RP>
constexpr size_t ring3_smem_bytes()
{
    return (size_t)(RP + 2) * Ring3Rows<Op, TY>::ROWS * RingGeomOf<Op>::WIDTH * sizeof(typename Op::T);
}

template <class Op, int TY3R, int RP3>
__global__ void __launch_bounds__(TY3R * 32) k_ring3d(FusedArgs a)
{
    extern __shared__ __align__(16) unsigned char s_ring_raw[];
    constexpr int RQ3 = RP3 + 2;
    using T = typename Op::T;
    using R = Ring3Rows<Op, TY3R>;
    constexpr int NV = Op::NV;
    constexpr int NR = Op::NR, NI = Op::NI;
    constexpr int VEC = RingGeomOf<Op>::VEC, STRIP = RingGeomOf<Op>::STRIP, OFF = RingGeomOf<Op>::OFF;
    constexpr int RWT = RingGeomOf<Op>::WIDTH;
    constexpr int SLOT = R::ROWS * RWT;
    Op op;
    if (op.skip(a)) return;
    op.begin(a);
    const Geom& g = a.g;
    T* ring = reinterpret_cast<T*>(s_ring_raw);
    const T* src_raw[NR];
    const T* src_in[NI > 0 ? NI : 1];
#pragma unroll
    for (int k = 0; k < NR; ++k) src_raw[k] = op.raw_ptr(a, k);
#pragma unroll
    for (int k = 0; k < NI; ++k) src_in[k] = op.in_ptr(a, k);
    const T* __restrict__ KX = op.coef_x(a);
    const T* __restrict__ KY = op.coef_y(a);
    const T* __restrict__ KZ = op.coef_z(a);
    DDVec<NV> acc;
    acc.zero();
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    const int xlast = g.X - HALO_PAD - 1;
    const int ylast = g.Y - HALO_PAD - 1;
    const int zlast = g.Z - HALO_PAD - 1;
    const int zlen = a.seg_rows;
    const int per_x = (g.nx + STRIP - 1) / STRIP;
    const int per_y = (g.ny + TY3R - 1) / TY3R;
    const long txy = (long)per_x * per_y;
    const long nunits = txy * ((g.nz + zlen - 1) / zlen);
    const int cmax = (int)g.pitch - 2 * VEC + 2;  // as in the 2D ring: copies stay inside the row
    for (long unit = blockIdx.x; unit < nunits; unit += gridDim.x) {
        const int zs = (int)(unit / txy);
        const long rxy = unit % txy;
        const int xs = (int)(rxy % per_x), ys = (int)(rxy / per_x);
        const int c0 = HALO_PAD + STRIP * xs;
        const int c = c0 + VEC * lane;
        const int cc = min(c, cmax);
        const int y0 = HALO_PAD + TY3R * ys;
        const int j = y0 + w;
        const bool row_active = j <= ylast;
        const int z0 = HALO_PAD + zlen * zs;
        const int z1 = min(z0 + zlen, zlast + 1);
        const int left = refl(c0 - 1, g.X);
        const int right_op = refl(min(c0 + STRIP, xlast + 1), g.X);
        const int right_k = min(c0 + STRIP, xlast + 1);
        // Operand rows are reflected into the inner domain, input rows clamped to the
        // boundary face row (Ky there is the face coefficient).
        const int rj = refl(min(j, ylast + 1), g.Y);
        const int ij = min(j, ylast + 1);
        const int r_below = refl(y0 - 1, g.Y);
        const int r_above = refl(min(y0 + TY3R, ylast + 1), g.Y);
        const int i_above = min(y0 + TY3R, ylast + 1);
        auto slot = [&](int z) { return ring + (size_t)((z - z0 + 1) % RQ3) * SLOT; };
        // Copy plane z of the tile: the operand rows for planes z0-1 .. z1, the rest for the
        // segment's planes, Kz also for plane z1 (the upper face of plane z1 - 1).
        auto issue = [&](int z) {
            if (z <= z1) {
                T* base = slot(z);
                const bool seg = z >= z0 && z < z1;
                const int zr = refl(min(z, zlast + 1), g.Z);
#pragma unroll
                for (int k = 0; k < NR; ++k) {
                    const T* sp = src_raw[k];
                    if (!sp) continue;
                    T* d = base + (R::RAW + k * (TY3R + 2)) * RWT;
                    cp_async_vecn<VEC>(d + (w + 1) * RWT + OFF + VEC * lane, sp + fidx(g, cc, rj, zr));
                    if (z >= z0) {
                        if (lane == 0) ring_copy_one(d + (w + 1) * RWT + OFF - 1, sp + fidx(g, left, rj, zr));
                        if (lane == 31)
                            ring_copy_one(d + (w + 1) * RWT + OFF + STRIP, sp + fidx(g, right_op, rj, zr));
                    }
                    if (seg && w == 0) cp_async_vecn<VEC>(d + OFF + VEC * lane, sp + fidx(g, cc, r_below, zr));
                    if (seg && w == TY3R - 1)
                        cp_async_vecn<VEC>(d + (TY3R + 1) * RWT + OFF + VEC * lane, sp + fidx(g, cc, r_above, zr));
                }
                if (seg) {
#pragma unroll
                    for (int k = 0; k < NI; ++k) {
                        if (!src_in[k]) continue;
                        cp_async_vecn<VEC>(base + (R::IN + k * TY3R + w) * RWT + OFF + VEC * lane,
                                           src_in[k] + fidx(g, cc, ij, z));
                    }
                    T* dx = base + (R::KX + w) * RWT;
                    cp_async_vecn<VEC>(dx + OFF + VEC * lane, KX + fidx(g, cc, ij, z));
                    if (lane == 31) ring_copy_one(dx + OFF + STRIP, KX + fidx(g, right_k, ij, z));
                    cp_async_vecn<VEC>(base + (R::KY + w) * RWT + OFF + VEC * lane, KY + fidx(g, cc, ij, z));
                    if (w == TY3R - 1)
                        cp_async_vecn<VEC>(base + (R::KY + TY3R) * RWT + OFF + VEC * lane, KY + fidx(g, cc, i_above, z));
                }
                if (z >= z0) cp_async_vecn<VEC>(base + (R::KZ + w) * RWT + OFF + VEC * lane, KZ + fidx(g, cc, ij, z));
            }
            cp_async_commit();
        };
        // The operand at slot row `row` (0 = the row below the tile) for the lane's cells.
        auto stage_row = [&](const T* base, int row, T* v) {
            T x[NR][VEC], xq[NR];
#pragma unroll
            for (int k = 0; k < NR; ++k) ld_vecn<VEC>(base + (R::RAW + k * (TY3R + 2) + row) * RWT + OFF + VEC * lane, x[k]);
#pragma unroll
            for (int q = 0; q < VEC; ++q) {
#pragma unroll
                for (int k = 0; k < NR; ++k) xq[k] = x[k][q];
                v[q] = op.stage_raw(op.raw_from(xq));
            }
        };
        // The operand at the strip's outside column of the warp's row (left for lane 0,
        // right for lane 31).
        auto stage_edge = [&](const T* base) {
            T xe[NR];
#pragma unroll
            for (int k = 0; k < NR; ++k)
                xe[k] = base[(R::RAW + k * (TY3R + 2) + w + 1) * RWT + (lane == 0 ? OFF - 1 : OFF + STRIP)];
            return op.stage_raw(op.raw_from(xe));
        };
        for (int z = z0 - 1; z <= z0 + RP3; ++z) issue(z);
        cp_async_wait<RP3>();
        __syncthreads();
        T mv[VEC], cv[VEC];
        stage_row(slot(z0 - 1), w + 1, mv);
        stage_row(slot(z0), w + 1, cv);
        T ce = stage_edge(slot(z0));
        for (int z = z0; z < z1; ++z) {
            cp_async_wait<RP3 - 1>();
            __syncthreads();
            issue(z + RP3 + 1);  // into the slot of plane z - 1, which no warp reads any more
            const T* cur = slot(z);
            const T* nxt = slot(z + 1);
            T pv[VEC], ym[VEC], yp[VEC];
            stage_row(nxt, w + 1, pv);
            const T pe = stage_edge(nxt);
            stage_row(cur, w, ym);
            stage_row(cur, w + 2, yp);
            const T up = __shfl_up_sync(0xffffffffu, cv[VEC - 1], 1);
            const T dn = __shfl_down_sync(0xffffffffu, cv[0], 1);
            T kx[VEC + 1], ky0[VEC], ky1[VEC], kz0[VEC], kz1[VEC];
            ld_vecn<VEC>(cur + (R::KX + w) * RWT + OFF + VEC * lane, kx);
            const T kxn = __shfl_down_sync(0xffffffffu, kx[0], 1);
            kx[VEC] = lane == 31 ? cur[(R::KX + w) * RWT + OFF + STRIP] : kxn;
            ld_vecn<VEC>(cur + (R::KY + w) * RWT + OFF + VEC * lane, ky0);
            ld_vecn<VEC>(cur + (R::KY + w + 1) * RWT + OFF + VEC * lane, ky1);
            ld_vecn<VEC>(cur + (R::KZ + w) * RWT + OFF + VEC * lane, kz0);
            ld_vecn<VEC>(nxt + (R::KZ + w) * RWT + OFF + VEC * lane, kz1);
            T rv[NR][VEC], iv[NI > 0 ? NI : 1][VEC];
#pragma unroll
            for (int k = 0; k < NR; ++k) ld_vecn<VEC>(cur + (R::RAW + k * (TY3R + 2) + w + 1) * RWT + OFF + VEC * lane, rv[k]);
#pragma unroll
            for (int k = 0; k < NI; ++k) ld_vecn<VEC>(cur + (R::IN + k * TY3R + w) * RWT + OFF + VEC * lane, iv[k]);
            auto cell_nb = [&](int q) {
                const int cq = c + q;
                NbT<T> nb;
                nb.c = cv[q];
                nb.xm = q == 0 ? (lane == 0 ? ce : up) : cv[q > 0 ? q - 1 : 0];
                nb.xp = cq == xlast ? cv[q] : (q == VEC - 1 ? (lane == 31 ? ce : dn) : cv[q < VEC - 1 ? q + 1 : q]);
                nb.ym = ym[q];
                nb.yp = yp[q];
                nb.zm = mv[q];
                nb.zp = pv[q];
                return nb;
            };
            if (row_active) {
                if constexpr (RingVecStore<Op>::value) {
                    typename Op::Out o[VEC];
#pragma unroll
                    for (int q = 0; q < VEC; ++q) {
                        T rq[NR], iq[NI > 0 ? NI : 1];
#pragma unroll
                        for (int k = 0; k < NR; ++k) rq[k] = rv[k][q];
#pragma unroll
                        for (int k = 0; k < NI; ++k) iq[k] = iv[k][q];
                        o[q] = op.interior_out(cell_nb(q), op.raw_from(rq), op.in_from(iq), kx[q], kx[q + 1], ky0[q],
                                               ky1[q], kz0[q], kz1[q], acc, c + q <= xlast);
                    }
                    const long i0 = fidx(g, c, j, z);
                    if (c + VEC - 1 <= xlast) {
                        op.store_vec(a, i0, o);
                    } else {
#pragma unroll
                        for (int q = 0; q < VEC; ++q)
                            if (c + q <= xlast) op.store_one(a, i0 + q, o[q]);
                    }
                } else {
#pragma unroll
                    for (int q = 0; q < VEC; ++q) {
                        const int cq = c + q;
                        if (cq <= xlast) {
                            T rq[NR], iq[NI > 0 ? NI : 1];
#pragma unroll
                            for (int k = 0; k < NR; ++k) rq[k] = rv[k][q];
#pragma unroll
                            for (int k = 0; k < NI; ++k) iq[k] = iv[k][q];
                            op.interior_k(a, fidx(g, cq, j, z), cell_nb(q), op.raw_from(rq), op.in_from(iq), kx[q],
                                          kx[q + 1], ky0[q], ky1[q], kz0[q], kz1[q], acc);
                        }
                    }
                }
            }
#pragma unroll
            for (int q = 0; q < VEC; ++q) {
                mv[q] = cv[q];
                cv[q] = pv[q];
            }
            ce = pe;
        }
        cp_async_wait<0>();
        __syncthreads();  // the next unit's copies reuse slots other warps may still read
    }
    if (Op::kReduce) grid_reduce_then<NV>(acc, a.red, [&](const double* v) { op.control(a, v); });
}
#endif

#if TEA_DIM == 2
#define TEA_STENCIL k_pipe2d
#define TEA_STENCIL_BLOCK dim3(SBLOCK)
#else
#define TEA_STENCIL k_pipe3d
#define TEA_STENCIL_BLOCK dim3(P3BLOCK)
#endif

// ------------------------------------------------------------------ CG / PPCG sweep A

// Applies the pending p update of the previous iteration (CGCalcP,
// tealeaf_2d/ext_cg_kernel.hpp:301-310, and for CG the deferred u += alpha p of CGCalcUr
// :251), then w = A p and pw = sum w.p (CGCalcW :177-189).  The new p goes to the other
// p buffer.
struct OpSweepA {
    static constexpr bool kReduce = true;
    using T = double;
    static constexpr int NV = 1;
    __device__ const double* coef_x(const FusedArgs& a) const { return a.kx; }
    __device__ const double* coef_y(const FusedArgs& a) const { return a.ky; }
    __device__ const double* coef_z(const FusedArgs& a) const { return a.kz; }
    const double* pcur;
    double* pnew;
    double beta, alpha;
    int pend_p, pend_u, precond;
    // An unrolled copy of the CG loop's body after the loop has ended (see enqueue_body).
    __device__ bool skip(const FusedArgs& a) { return a.st->cont == 0; }
    __device__ void begin(const FusedArgs& a)
    {
        const SolveState& s = *a.st;
        pcur = a.p[s.par_p];
        pnew = a.p[s.par_p ^ 1];
        beta = s.last_beta;
        alpha = s.last_alpha;
        pend_p = s.pending_p;
        pend_u = s.pending_u;
        precond = s.precond;
    }
    // Pipelined 2D interface (k_pipe2d): raw loads, staging, interior from registers.
    struct Raw {
        double p, q;
    };
    struct In {
        double u;
    };
    __device__ Raw load_raw(const FusedArgs& a, long i) const
    {
        Raw r;
        r.p = pcur[i];
        r.q = pend_p ? (precond ? a.z[i] : a.r[i]) : 0.0;
        return r;
    }
    __device__ double stage_raw(const Raw& r) const { return pend_p ? beta * r.p + r.q : r.p; }
    __device__ In load_in(const FusedArgs& a, long i) const
    {
        In in;
        in.u = pend_u ? a.u[0][i] : 0.0;
        return in;
    }
    // Ring interface (k_ring2d): the arrays behind Raw and In, and Raw/In from their values.
    static constexpr int NR = 2, NI = 1;
    __device__ const double* raw_ptr(const FusedArgs& a, int k) const
    {
        return k == 0 ? pcur : (pend_p ? (precond ? a.z : a.r) : nullptr);
    }
    __device__ const double* in_ptr(const FusedArgs& a, int) const { return pend_u ? a.u[0] : nullptr; }
    __device__ Raw raw_from(const double* v) const
    {
        Raw r;
        r.p = v[0];
        r.q = pend_p ? v[1] : 0.0;
        return r;
    }
    __device__ In in_from(const double* v) const
    {
        In in;
        in.u = pend_u ? v[0] : 0.0;
        return in;
    }
    __device__ void interior_k(const FusedArgs& a, long i, const Nb& nb, const Raw& rc, const In& in, double kx0,
                               double kx1, double ky0, double ky1, double kz0, double kz1, DDVec<1>& acc) const
    {
        if (pend_u) a.u[0][i] = in.u + alpha * rc.p;
        pnew[i] = nb.c;
        const double w = smvp_k(nb, kx0, kx1, ky0, ky1, kz0, kz1);
        a.w[i] = w;
        dd_add(acc.v[0], w * nb.c);
    }
    __device__ void control(const FusedArgs& a, const double* v)
    {
        const double pw = v[0];
        if (a.timing) return;
        SolveState& s = *a.st;
        s.pw = pw;
        s.alpha = s.rro / pw;
        a.cg_alphas[s.n] = s.alpha;
        s.par_p ^= 1;
        s.pending_p = 0;
        s.pending_u = 0;
        if (!isfinite(pw)) s.nonfinite = 1;
    }
};

// ------------------------------------------------------------------ CG sweep B

// Pointwise sweeps walk the inner domain in row segments of 64 cells: each warp takes a
// segment, each lane two adjacent cells with 16-byte loads and stores (the first inner
// cell of every row is 256-byte aligned, so kk = 2 + 2*lane is 16-byte aligned).
struct Seg {
    long nseg;   // segments in the inner domain
    int per_row;
};

__host__ __device__ inline Seg make_seg(const Geom& g)
{
    Seg s;
    s.per_row = (g.nx + 63) / 64;
    s.nseg = (long)s.per_row * g.ny * g.nz;
    return s;
}

template <class F>
__device__ __forceinline__ void walk_pairs(const Geom& g, F&& f)
{
    const Seg sg = make_seg(g);
    const int lane = threadIdx.x & 31;
    const long warp0 = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long nwarps = ((long)gridDim.x * blockDim.x) >> 5;
    const int xlast = g.X - HALO_PAD - 1;
    for (long sgi = warp0; sgi < sg.nseg; sgi += nwarps) {
        const long row = sgi / sg.per_row;
        const int xs = (int)(sgi - row * sg.per_row);
        const int jj = HALO_PAD + (int)(row % g.ny);
        const int ii = DIM == 3 ? HALO_PAD + (int)(row / g.ny) : 0;
        const int kk = HALO_PAD + xs * 64 + 2 * lane;
        if (kk <= xlast) f(fidx(g, kk, jj, ii), kk < xlast);
    }
}

// FP32 variant of walk_pairs: 128-cell row segments, four adjacent cells per lane (one
// 16-byte access); f(i, n) gets the first cell and how many of the four are inner (1..4).
template <class F>
__device__ __forceinline__ void walk_quads(const Geom& g, F&& f)
{
    const int per_row = (g.nx + 127) / 128;
    const long nseg = (long)per_row * g.ny * g.nz;
    const int lane = threadIdx.x & 31;
    const long warp0 = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long nwarps = ((long)gridDim.x * blockDim.x) >> 5;
    const int xlast = g.X - HALO_PAD - 1;
    for (long sgi = warp0; sgi < nseg; sgi += nwarps) {
        const long row = sgi / per_row;
        const int xs = (int)(sgi - row * per_row);
        const int jj = HALO_PAD + (int)(row % g.ny);
        const int ii = DIM == 3 ? HALO_PAD + (int)(row / g.ny) : 0;
        const int kk = HALO_PAD + xs * 128 + 4 * lane;
        if (kk <= xlast) f(fidx(g, kk, jj, ii), min(4, xlast - kk + 1));
    }
}

__device__ __forceinline__ double2 ld2(const double* p) { return *reinterpret_cast<const double2*>(p); }
__device__ __forceinline__ void st2(double* p, double a, double b) { *reinterpret_cast<double2*>(p) = make_double2(a, b); }

// CGCalcUr without the u update (deferred to the next sweep A): r -= alpha w, z = Mi r,
// rrn = sum r.r or r.z; then beta = rrn/rro and the end-of-iteration test.
__global__ void __launch_bounds__(256) k_cg_sweep_b(FusedArgs a)
{
    if (a.st->cont == 0) return;  // an unrolled copy after the loop has ended (uniform)
    const SolveState& s = *a.st;
    const double alpha = s.alpha;
    const int precond = s.precond;
    double* __restrict__ R = a.r;
    const double* __restrict__ W = a.w;
    const double* __restrict__ MI = a.mi;
    double* __restrict__ Z = a.z;
    DDVec<1> acc;
    acc.zero();
    walk_pairs(a.g, [&](long i, bool two) {
        if (two) {
            const double2 r2 = ld2(R + i), w2 = ld2(W + i);
            const double r0 = r2.x - alpha * w2.x, r1 = r2.y - alpha * w2.y;
            st2(R + i, r0, r1);
            if (precond) {
                const double2 m2 = ld2(MI + i);
                const double z0 = m2.x * r0, z1 = m2.y * r1;
                st2(Z + i, z0, z1);
                dd_add(acc.v[0], r0 * z0);
                dd_add(acc.v[0], r1 * z1);
            } else {
                dd_add(acc.v[0], r0 * r0);
                dd_add(acc.v[0], r1 * r1);
            }
        } else {
            const double r0 = R[i] - alpha * W[i];
            R[i] = r0;
            if (precond) {
                const double z0 = MI[i] * r0;
                Z[i] = z0;
                dd_add(acc.v[0], r0 * z0);
            } else {
                dd_add(acc.v[0], r0 * r0);
            }
        }
    });
    grid_reduce_then<1>(acc, a.red, [&](const double* v) {
        if (a.timing) return;
        SolveState& st = *a.st;
        st.rrn = v[0];
        st.beta = st.rrn / st.rro;
        a.cg_betas[st.n] = st.beta;
        st.error = st.rrn;
        st.rro = st.rrn;
        st.last_alpha = st.alpha;
        st.last_beta = st.beta;
        st.pending_p = 1;
        st.pending_u = 1;
        if (!isfinite(v[0])) st.nonfinite = 1;
        end_iteration(a, st, PHASE_CG);
    });
}

// ------------------------------------------------------------------ PPCG

// CGCalcUr (u += alpha p, r -= alpha w, z = Mi r; its rrn is unused,
// tealeaf_2d/tea_solve.f90:340) fused with PPCGInitSd (tealeaf_2d/ext_ppcg_kernel.hpp:8-34)
// writing sd into buffer 0.
__global__ void __launch_bounds__(256) k_ppcg_sweep_b(FusedArgs a)
{
    const SolveState& s = *a.st;
    const double alpha = s.alpha, theta = s.theta;
    const int precond = s.precond;
    const double* __restrict__ p = a.p[s.par_p];
    double* __restrict__ U = a.u[0];
    const double* R = a.r;
    const double* W = a.w;
    double* RD = a.r_in_w ? a.w : a.r;  // where r goes: w when the two-step passes start there
    double* __restrict__ SD = a.sd[0];
    walk_pairs(a.g, [&](long i, bool two) {
        if (two) {
            const double2 u2 = ld2(U + i), p2 = ld2(p + i), r2 = ld2(R + i), w2 = ld2(W + i);
            st2(U + i, u2.x + alpha * p2.x, u2.y + alpha * p2.y);
            const double r0 = r2.x - alpha * w2.x, r1 = r2.y - alpha * w2.y;
            st2(RD + i, r0, r1);
            double m0 = r0, m1 = r1;
            if (precond) {
                const double2 mi = ld2(a.mi + i);
                m0 = mi.x * r0;
                m1 = mi.y * r1;
                st2(a.z + i, m0, m1);
            }
            st2(SD + i, m0 / theta, m1 / theta);
        } else {
            U[i] = U[i] + alpha * p[i];
            const double r = R[i] - alpha * W[i];
            RD[i] = r;
            double m = r;
            if (precond) {
                m = a.mi[i] * r;
                a.z[i] = m;
            }
            SD[i] = m / theta;
        }
    });
}

// One PPCG inner step k (1-based): PPCGCalcU (r -= A sd, u += sd,
// tealeaf_2d/ext_ppcg_kernel.hpp:37-65) then PPCGCalcSd (:68-100) into the other sd
// buffer.  The last step also forms sum r.r (ext_calculate_2norm_, tea_solve.f90:346)
// and runs the end of the outer iteration (beta, calc_p deferred, EXIT test).
template <bool LAST>
struct OpPPCGInner {
    static constexpr bool kReduce = LAST;
    using T = double;
    static constexpr int NV = 1;
    __device__ const double* coef_x(const FusedArgs& a) const { return a.kx; }
    __device__ const double* coef_y(const FusedArgs& a) const { return a.ky; }
    __device__ const double* coef_z(const FusedArgs& a) const { return a.kz; }
    const double* sdc;
    double* sdn;
    double al, be;
    int precond;
    int k;
    __device__ bool skip(const FusedArgs&) { return false; }
    __device__ void begin(const FusedArgs& a)
    {
        k = a.step;
        const SolveState& s = *a.st;
        sdc = a.sd[(k - 1) & 1];
        sdn = a.sd[k & 1];
        al = a.ch_alphas[k - 1];
        be = a.ch_betas[k - 1];
        precond = s.precond;
    }
    struct Raw {
        double sd;
    };
    struct In {
        double r, u, mi;
    };
    __device__ Raw load_raw(const FusedArgs&, long i) const
    {
        Raw r;
        r.sd = sdc[i];
        return r;
    }
    __device__ double stage_raw(const Raw& r) const { return r.sd; }
    __device__ In load_in(const FusedArgs& a, long i) const
    {
        In in;
        in.r = a.r[i];
        in.u = a.u[0][i];
        in.mi = precond ? a.mi[i] : 0.0;
        return in;
    }
    static constexpr int NR = 1, NI = 3;
    __device__ const double* raw_ptr(const FusedArgs&, int) const { return sdc; }
    __device__ const double* in_ptr(const FusedArgs& a, int k) const
    {
        return k == 0 ? a.r : (k == 1 ? a.u[0] : (precond ? a.mi : nullptr));
    }
    __device__ Raw raw_from(const double* v) const
    {
        Raw r;
        r.sd = v[0];
        return r;
    }
    __device__ In in_from(const double* v) const
    {
        In in;
        in.r = v[0];
        in.u = v[1];
        in.mi = precond ? v[2] : 0.0;
        return in;
    }
    __device__ void interior_k(const FusedArgs& a, long i, const Nb& nb, const Raw&, const In& in, double kx0,
                               double kx1, double ky0, double ky1, double kz0, double kz1, DDVec<1>& acc) const
    {
        const double s = smvp_k(nb, kx0, kx1, ky0, ky1, kz0, kz1);
        const double r = in.r - s;
        a.r[i] = r;
        a.u[0][i] = in.u + nb.c;
        sdn[i] = al * nb.c + be * (precond ? in.mi * r : r);
        if (LAST) dd_add(acc.v[0], r * r);
    }
    __device__ void control(const FusedArgs& a, const double* v)
    {
        const double rrn = v[0];
        if (a.timing) return;
        SolveState& s = *a.st;
        s.rrn = rrn;
        s.beta = s.rrn / s.rro;
        s.error = s.rrn;
        s.rro = s.rrn;
        s.last_beta = s.beta;
        s.pending_p = 1;
        s.pending_u = 0;
        s.cheby_calc_steps = s.cheby_calc_steps + 1;
        if (!isfinite(rrn)) s.nonfinite = 1;
        end_iteration(a, s, PHASE_PPCG);
    }
};

// Arrays, scalars and end of the outer iteration of the two-step PPCG pass: the FP64
// solve's (PpcgF64), or the FP32 inner PPCG of the defect-correction form (PpcgF32: the
// correction d in place of u, FP32 r, w, sd and coefficients, no preconditioner).
struct PpcgF64 {
    using T = double;
    __device__ static T* sd(const FusedArgs& a, int b) { return a.sd[b]; }
    __device__ static T* r(const FusedArgs& a) { return a.r; }
    __device__ static T* w(const FusedArgs& a) { return a.w; }
    __device__ static T* u(const FusedArgs& a) { return a.u[0]; }
    __device__ static const T* mi(const FusedArgs& a) { return a.st->precond ? a.mi : nullptr; }
    __device__ static const T* kx(const FusedArgs& a) { return a.kx; }
    __device__ static const T* ky(const FusedArgs& a) { return a.ky; }
    __device__ static const T* kz(const FusedArgs& a) { return a.kz; }
    __device__ static void control(const FusedArgs& a, const double* v) { OpPPCGInner<true>().control(a, v); }
};
struct PpcgF32 {
    using T = float;
    __device__ static T* sd(const FusedArgs& a, int b) { return a.sd32[b]; }
    __device__ static T* r(const FusedArgs& a) { return a.r32; }
    __device__ static T* w(const FusedArgs& a) { return a.w32; }
    __device__ static T* u(const FusedArgs& a) { return a.d32; }
    __device__ static const T* mi(const FusedArgs&) { return nullptr; }
    __device__ static const T* kx(const FusedArgs& a) { return a.kx32; }
    __device__ static const T* ky(const FusedArgs& a) { return a.ky32; }
    __device__ static const T* kz(const FusedArgs& a) { return a.kz32; }
    // End of an inner PPCG iteration: beta for the next p = r + beta p (applied by the FP32
    // sweep A), and the inner loop test of the FP32 CG (stop below tol2 or at inner_max).
    __device__ static void control(const FusedArgs& a, const double* v)
    {
        if (a.timing) return;
        SolveState& s = *a.st;
        const double rrn = v[0];
        s.rrn = rrn;
        s.beta = rrn / s.rro;
        s.rro = rrn;
        s.last_beta = s.beta;
        s.pending_p = 1;
        s.pending_u = 0;
        s.n_inner = s.n_inner + 1;
        if (!isfinite(rrn)) s.inner_diverged = 1;  // the correction is dropped; CG takes over
        const int cont = isfinite(rrn) && rrn >= s.tol2 && s.n_inner < s.inner_max;
        s.cont = cont;
        if (a.use_handle) cudaGraphSetConditional(a.handle, cont ? 1u : 0u);
    }
};

#if TEA_DIM == 3
// Two PPCG inner steps k, k+1 in one pass over the 3D field (temporal blocking).  The
// reference refreshes sd's halo by reflection before every inner step
// (tealeaf_2d/tea_solve.f90:631-636) and the steps between the outer iteration's sweeps
// have no reduction except on the last one, so two of them share one read of sd, r, u, mi
// and K and one write of r, u and sd: about 9 words per cell for two steps instead of
// eighteen.  Per cell the operations and their order are those of two single steps, so the
// results are bit-identical.
//
// The plane ring of k_ring3d (a block of TY warps, a 64-column x TY-row tile marching
// through a z segment) computes step k for every loaded cell one plane ahead of step k+1.
// Step k+1 needs step k's sd at its neighbours: z-neighbours stay in registers, y-neighbours
// go through a two-plane shared buffer, x-neighbours by shuffle.  So a tile writes only its
// inner 60 columns (lanes 1..30) and rows (warps 1..TY-2): tiles overlap by four columns and
// two rows, z segments by one plane of step k.  At the domain's faces step k's sd is
// reflected as the reference's halo update reflects it (the cell's own value).  Tiles read
// r at cells that a neighbouring tile writes, so r goes to the other of r and w (w is free
// during the inner steps) and sd to the other sd buffer.  Pair m (steps 2m-1, 2m) reads
// sd[(m-1)&1] and writes sd[m&1]; it reads r from r when m - 1 + a.r_in_w is even, else from
// w, and writes it to the other.  With an odd number of pairs sweep B leaves r in w
// (r_in_w), so the last pair writes r back into r.  A pair whose second step is the last
// inner step also forms that step's sum r.r and ends the outer iteration.
//
// A ring slot holds, per plane, the tile's rows of each input and nothing outside the strip
// (x-neighbours come by shuffle), and the preconditioner's rows only in the PRE form: without
// them a slot of TY = 8 is 51 rows of 512 bytes, so that with one plane in flight (RP = 1)
// two blocks fit on an SM.
template <int TY, bool PRE>
struct Ppcg2Rows {
    static constexpr int RAW = 0;                      // sd: TY + 2 rows
    static constexpr int IN_R = TY + 2;                // r
    static constexpr int IN_U = IN_R + TY;             // u
    static constexpr int IN_MI = IN_U + TY;            // mi (PRE only)
    static constexpr int KX = IN_MI + (PRE ? TY : 0);  // TY
    static constexpr int KY = KX + TY;                 // TY + 1
    static constexpr int KZ = KY + TY + 1;             // TY
    static constexpr int ROWS = KZ + TY;
};

template <class T, int TY, int RP, bool PRE>
constexpr size_t ppcg2_smem_bytes()
{
    return (size_t)(RP + 3) * Ppcg2Rows<TY, PRE>::ROWS * RingGeom<T>::STRIP * sizeof(T)
        + (size_t)2 * TY * RingGeom<T>::STRIP * sizeof(T);
}

template <class P, int TY, int RP, bool PRE>
__global__ void __launch_bounds__(TY * 32) k_ppcg2_ring3d(FusedArgs a)
{
    using T = typename P::T;
    extern __shared__ __align__(16) unsigned char s_raw[];
    using R = Ppcg2Rows<TY, PRE>;
    constexpr int VEC = RingGeom<T>::VEC, STRIP = RingGeom<T>::STRIP, OFF = 0;
    constexpr int RWT = STRIP;
    constexpr int OUT = 30 * VEC;
    constexpr int RQ = RP + 3;
    constexpr int SLOT = R::ROWS * RWT;
    constexpr int IN_R = R::IN_R, IN_U = R::IN_U, IN_MI = R::IN_MI;
    T* ring = reinterpret_cast<T*>(s_raw);
    T* s1 = ring + (size_t)RQ * SLOT;  // step k's sd: [plane parity][TY rows][STRIP]
    const Geom& g = a.g;
    const int k = a.step;
    const int m = (k + 1) >> 1;
    const T* __restrict__ sdk = P::sd(a, (m - 1) & 1);
    T* __restrict__ sdo = P::sd(a, m & 1);
    const T* __restrict__ rin = ((m - 1 + a.r_in_w) & 1) ? P::w(a) : P::r(a);
    T* __restrict__ rout = ((m + a.r_in_w) & 1) ? P::w(a) : P::r(a);
    T* __restrict__ U = P::u(a);
    const T* __restrict__ MI = PRE ? P::mi(a) : nullptr;
    const bool precond = PRE && MI != nullptr;
    const bool last = k + 1 == a.st->inner_steps;  // step k+1 ends the outer iteration
    DDVec<1> acc;
    acc.zero();
    const T al1 = (T)a.ch_alphas[k - 1], be1 = (T)a.ch_betas[k - 1];
    const T al2 = (T)a.ch_alphas[k], be2 = (T)a.ch_betas[k];
    const T* __restrict__ KX = P::kx(a);
    const T* __restrict__ KY = P::ky(a);
    const T* __restrict__ KZ = P::kz(a);
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    const int xlast = g.X - HALO_PAD - 1;
    const int ylast = g.Y - HALO_PAD - 1;
    const int zlast = g.Z - HALO_PAD - 1;
    const int zlen = a.seg_rows;
    const int per_x = (g.nx + OUT - 1) / OUT;
    const int per_y = (g.ny + TY - 3) / (TY - 2);
    const long txy = (long)per_x * per_y;
    const long nunits = txy * ((g.nz + zlen - 1) / zlen);
    const int cmax = (int)g.pitch - 2 * VEC + 2;
    const bool lane_out = lane >= 1 && lane <= 30;
    for (long unit = blockIdx.x; unit < nunits; unit += gridDim.x) {
        const int zs = (int)(unit / txy);
        const long rxy = unit % txy;
        const int xs = (int)(rxy % per_x), ys = (int)(rxy / per_x);
        const int c = HALO_PAD - VEC + OUT * xs + VEC * lane;  // >= 0: lane 0 of strip 0 sits on the halo
        const int cc = min(c, cmax);
        const int y0 = HALO_PAD - 1 + (TY - 2) * ys;
        const int j = y0 + w;
        const bool row_in = j >= HALO_PAD && j <= ylast;              // step k computed
        const bool row_out = w >= 1 && w <= TY - 2 && j <= ylast;     // step k+1 written
        const int z0 = HALO_PAD + zlen * zs;
        const int z1 = min(z0 + zlen, zlast + 1);
        const int zf = z0 > HALO_PAD ? z0 - 1 : z0;  // first plane of step k
        const int zl = min(z1, zlast);              // last plane of step k
        const int rj = refl(min(j, ylast + 1), g.Y);
        const int ij = min(max(j, HALO_PAD), ylast + 1);
        const int r_below = refl(y0 - 1, g.Y);
        const int r_above = refl(min(y0 + TY, ylast + 1), g.Y);
        const int i_above = min(y0 + TY, ylast + 1);
        auto slot = [&](int p) { return ring + (size_t)((p - zf + 1) % RQ) * SLOT; };
        // Plane p of the tile: sd at the warps' rows for planes zf-1 .. zl+1, the rest for
        // step k's planes, Kz also for plane zl+1.
        auto issue = [&](int p) {
            if (p <= zl + 1) {
                T* base = slot(p);
                const int pr = refl(min(p, zlast + 1), g.Z);
                const int pi = min(p, zlast + 1);
                const int col = OFF + VEC * lane;
                cp_async_16(base + (R::RAW + w + 1) * RWT + col, sdk + fidx(g, cc, rj, pr));
                if (p >= zf && p <= zl) {
                    if (w == 0) cp_async_16(base + R::RAW * RWT + col, sdk + fidx(g, cc, r_below, pr));
                    if (w == TY - 1) cp_async_16(base + (R::RAW + TY + 1) * RWT + col, sdk + fidx(g, cc, r_above, pr));
                    cp_async_16(base + (IN_R + w) * RWT + col, rin + fidx(g, cc, ij, pi));
                    if (row_out && lane_out) cp_async_16(base + (IN_U + w) * RWT + col, U + fidx(g, cc, ij, pi));
                    if (PRE && MI) cp_async_16(base + (IN_MI + w) * RWT + col, MI + fidx(g, cc, ij, pi));
                    cp_async_16(base + (R::KX + w) * RWT + col, KX + fidx(g, cc, ij, pi));
                    cp_async_16(base + (R::KY + w) * RWT + col, KY + fidx(g, cc, ij, pi));
                    if (w == TY - 1) cp_async_16(base + (R::KY + TY) * RWT + col, KY + fidx(g, cc, i_above, pi));
                }
                if (p >= zf) cp_async_16(base + (R::KZ + w) * RWT + col, KZ + fidx(g, cc, ij, pi));
            }
            cp_async_commit();
        };
        auto own = [&](const T* base, int row, T* v) { ld_vec(base + row * RWT + OFF + VEC * lane, v); };
        // Step k at plane p from sd at planes p-1 (A), p (B), p+1 (C): r1, u1 and sd1 at the
        // lane's cells; sd1 also into the shared plane buffer.
        auto step1 = [&](int p, const T* A, const T* B, const T* C, T* r1, T* u1, T* t1) {
            const T* cur = slot(p);
            const T* nxt = slot(p + 1);
            const T up = __shfl_up_sync(0xffffffffu, B[VEC - 1], 1);
            const T dn = __shfl_down_sync(0xffffffffu, B[0], 1);
            T kx[VEC + 1];
            own(cur, R::KX + w, kx);
            kx[VEC] = __shfl_down_sync(0xffffffffu, kx[0], 1);
            if (p <= zl && row_in) {
                T ky0[VEC], ky1[VEC], kz0[VEC], kz1[VEC], ym[VEC], yp[VEC], rr[VEC], uu[VEC], mi[VEC];
                own(cur, R::KY + w, ky0);
                own(cur, R::KY + w + 1, ky1);
                own(cur, R::KZ + w, kz0);
                own(nxt, R::KZ + w, kz1);
                own(cur, R::RAW + w, ym);
                own(cur, R::RAW + w + 2, yp);
                own(cur, IN_R + w, rr);
                own(cur, IN_U + w, uu);
                if (precond) own(cur, IN_MI + w, mi);
#pragma unroll
                for (int q = 0; q < VEC; ++q) {
                    NbT<T> nb;
                    nb.c = B[q];
                    nb.xm = c + q == HALO_PAD ? B[q] : (q == 0 ? up : B[q > 0 ? q - 1 : 0]);
                    nb.xp = c + q == xlast ? B[q] : (q == VEC - 1 ? dn : B[q < VEC - 1 ? q + 1 : q]);
                    nb.ym = ym[q];
                    nb.yp = yp[q];
                    nb.zm = A[q];
                    nb.zp = C[q];
                    const T s = smvp_k(nb, kx[q], kx[q + 1], ky0[q], ky1[q], kz0[q], kz1[q]);
                    const T r = rr[q] - s;
                    r1[q] = r;
                    u1[q] = uu[q] + B[q];
                    t1[q] = al1 * B[q] + be1 * (precond ? mi[q] * r : r);
                }
            } else {
#pragma unroll
                for (int q = 0; q < VEC; ++q) r1[q] = u1[q] = t1[q] = (T)0;
            }
            st_vec(s1 + ((size_t)(p & 1) * TY + w) * STRIP + VEC * lane, t1);
        };
        for (int p = zf - 1; p < zf - 1 + RQ; ++p) issue(p);
        cp_async_wait<RQ - 3>();
        __syncthreads();
        T sA[VEC], sB[VEC], sC[VEC];  // sd at planes z, z+1, z+2 (the warp's row)
        T tm[VEC], tc[VEC], tn[VEC];  // step k's sd at planes z-1, z, z+1
        T r1c[VEC], u1c[VEC], r1n[VEC], u1n[VEC];
        {
            T sM[VEC];
            own(slot(zf - 1), R::RAW + w + 1, sM);
            own(slot(zf), R::RAW + w + 1, sA);
            own(slot(zf + 1), R::RAW + w + 1, sB);
            step1(zf, sM, sA, sB, r1c, u1c, tc);
#pragma unroll
            for (int q = 0; q < VEC; ++q) tm[q] = tc[q];
        }
        for (int z = zf; z < z1; ++z) {
            cp_async_wait<RP - 1>();
            __syncthreads();
            issue(z + RP + 2);  // into the slot of plane z - 1, which no warp reads any more
            own(slot(z + 2), R::RAW + w + 1, sC);
            step1(z + 1, sA, sB, sC, r1n, u1n, tn);
            if (z >= z0) {
                // Step k+1 at plane z.
                const T* cur = slot(z);
                const T* nxt = slot(z + 1);
                const T up = __shfl_up_sync(0xffffffffu, tc[VEC - 1], 1);
                const T dn = __shfl_down_sync(0xffffffffu, tc[0], 1);
                T kx[VEC + 1];
                own(cur, R::KX + w, kx);
                kx[VEC] = __shfl_down_sync(0xffffffffu, kx[0], 1);
                if (row_out && lane_out) {
                    T ky0[VEC], ky1[VEC], kz0[VEC], kz1[VEC], ym[VEC], yp[VEC], mi[VEC];
                    own(cur, R::KY + w, ky0);
                    own(cur, R::KY + w + 1, ky1);
                    own(cur, R::KZ + w, kz0);
                    own(nxt, R::KZ + w, kz1);
                    if (precond) own(cur, IN_MI + w, mi);
                    const T* sp = s1 + (size_t)(z & 1) * TY * STRIP + VEC * lane;
                    if (j > HALO_PAD) ld_vec(sp + (w - 1) * STRIP, ym);
                    if (j < ylast) ld_vec(sp + (w + 1) * STRIP, yp);
                    T r2[VEC], u2[VEC], d2[VEC];
#pragma unroll
                    for (int q = 0; q < VEC; ++q) {
                        NbT<T> nb;
                        nb.c = tc[q];
                        nb.xm = c + q == HALO_PAD ? tc[q] : (q == 0 ? up : tc[q > 0 ? q - 1 : 0]);
                        nb.xp = c + q == xlast ? tc[q] : (q == VEC - 1 ? dn : tc[q < VEC - 1 ? q + 1 : q]);
                        nb.ym = j == HALO_PAD ? tc[q] : ym[q];
                        nb.yp = j == ylast ? tc[q] : yp[q];
                        nb.zm = z == HALO_PAD ? tc[q] : tm[q];
                        nb.zp = z == zlast ? tc[q] : tn[q];
                        const T s = smvp_k(nb, kx[q], kx[q + 1], ky0[q], ky1[q], kz0[q], kz1[q]);
                        const T r = r1c[q] - s;
                        r2[q] = r;
                        u2[q] = u1c[q] + tc[q];
                        d2[q] = al2 * tc[q] + be2 * (precond ? mi[q] * r : r);
                        if (last && c + q <= xlast) dd_add(acc.v[0], (double)r * (double)r);
                    }
                    const long i = fidx(g, c, j, z);
                    if (c + VEC - 1 <= xlast) {
                        st_vec(rout + i, r2);
                        st_vec(U + i, u2);
                        st_vec(sdo + i, d2);
                    } else {
#pragma unroll
                        for (int q = 0; q < VEC; ++q) {
                            if (c + q <= xlast) {
                                rout[i + q] = r2[q];
                                U[i + q] = u2[q];
                                sdo[i + q] = d2[q];
                            }
                        }
                    }
                }
            }
#pragma unroll
            for (int q = 0; q < VEC; ++q) {
                sA[q] = sB[q];
                sB[q] = sC[q];
                tm[q] = tc[q];
                tc[q] = tn[q];
                r1c[q] = r1n[q];
                u1c[q] = u1n[q];
            }
        }
        cp_async_wait<0>();
        __syncthreads();  // the next unit's copies reuse slots other warps may still read
    }
    // The last inner step's sum r.r and the end of the outer iteration.
    if (last) grid_reduce_then<1>(acc, a.red, [&](const double* v) { P::control(a, v); });
}
#endif

// ------------------------------------------------------------------ Chebyshev

// ChebyIterate + ChebyCalcU (tealeaf_2d/ext_cheby_kernel.hpp:50-115) in one sweep: the
// operator reads u_old, u_new = u_old + p goes to the other u buffer.  sum r.r is formed
// on the iterations where tea_leaf() checks it (n >= est_itc and MOD(n,10) == 0,
// tealeaf_2d/tea_solve.f90:260).
struct OpCheby {
    static constexpr bool kReduce = true;
    using T = double;
    static constexpr int NV = 1;
    __device__ const double* coef_x(const FusedArgs& a) const { return a.kx; }
    __device__ const double* coef_y(const FusedArgs& a) const { return a.ky; }
    __device__ const double* coef_z(const FusedArgs& a) const { return a.kz; }
    const double* ucur;
    double* unew;
    double* pcur;  // p is updated in place (pointwise); the two-iteration kernel ping-pongs it
    double* pnext;
    double al, be;
    int precond, check;
    __device__ bool skip(const FusedArgs&) { return false; }
    __device__ void begin(const FusedArgs& a)
    {
        const SolveState& s = *a.st;
        ucur = a.u[s.par_u];
        unew = a.u[s.par_u ^ 1];
        pcur = a.p[s.par_p];
        pnext = a.p[s.par_p ^ 1];
        const int step = s.cheby_calc_steps - 1;
        al = a.ch_alphas[step];
        be = a.ch_betas[step];
        precond = s.precond;
        check = (s.n >= s.est_itc) && (s.n % 10 == 0);
    }
    struct Raw {
        double u;
    };
    struct In {
        double u0, p, mi;
    };
    __device__ Raw load_raw(const FusedArgs&, long i) const
    {
        Raw r;
        r.u = ucur[i];
        return r;
    }
    __device__ double stage_raw(const Raw& r) const { return r.u; }
    __device__ In load_in(const FusedArgs& a, long i) const
    {
        In in;
        in.u0 = a.u0[i];
        in.p = pcur[i];
        in.mi = precond ? a.mi[i] : 0.0;
        return in;
    }
    static constexpr int NR = 1, NI = 3;
    __device__ const double* raw_ptr(const FusedArgs&, int) const { return ucur; }
    __device__ const double* in_ptr(const FusedArgs& a, int k) const
    {
        return k == 0 ? a.u0 : (k == 1 ? pcur : (precond ? a.mi : nullptr));
    }
    __device__ Raw raw_from(const double* v) const
    {
        Raw r;
        r.u = v[0];
        return r;
    }
    __device__ In in_from(const double* v) const
    {
        In in;
        in.u0 = v[0];
        in.p = v[1];
        in.mi = precond ? v[2] : 0.0;
        return in;
    }
    __device__ void interior_k(const FusedArgs& a, long i, const Nb& nb, const Raw&, const In& in, double kx0,
                               double kx1, double ky0, double ky1, double kz0, double kz1, DDVec<1>& acc) const
    {
        const double w = smvp_k(nb, kx0, kx1, ky0, ky1, kz0, kz1);
        const double r = in.u0 - w;
        const double p = al * in.p + be * (precond ? in.mi * r : r);
        pcur[i] = p;
        unew[i] = nb.c + p;
        if (check) dd_add(acc.v[0], r * r);
    }
    __device__ void control(const FusedArgs& a, const double* v)
    {
        const double rr = v[0];
        if (a.timing) return;
        SolveState& s = *a.st;
        s.par_u ^= 1;
        if (check) s.error = rr;
        s.cheby_calc_steps = s.cheby_calc_steps + 1;
        end_iteration(a, s, PHASE_CHEBY);
    }
    // Passes of nit iterations (k_cheby2_ring2d, k_cheby4_ring2d): a pass runs unless one of
    // its first nit - 1 iterations is a convergence check (which must end a launch) or it
    // would go past max_iters.
    __device__ bool pass_ok(const FusedArgs& a, int nit) const
    {
        const SolveState& st = *a.st;
        for (int k = 0; k < nit - 1; ++k) {
            const int it = st.n + k;
            if (it >= st.est_itc && it % 10 == 0) return false;
        }
        return st.n + nit - 1 <= st.max_iters;
    }
    // Coefficients of the pass's iteration l (0-based).
    __device__ void pass_coefs(const FusedArgs& a, int l, double& al_l, double& be_l) const
    {
        const int k = a.st->cheby_calc_steps - 1 + l;
        al_l = a.ch_alphas[k];
        be_l = a.ch_betas[k];
    }
    __device__ bool pass_check(const FusedArgs& a, int nit) const
    {
        const SolveState& st = *a.st;
        const int it = st.n + nit - 1;
        return it >= st.est_itc && it % 10 == 0;
    }
    __device__ const double* pair_rhs(const FusedArgs& a) const { return a.u0; }
    __device__ const double* pair_mi(const FusedArgs& a) const { return precond ? a.mi : nullptr; }
    __device__ void pass_control(const FusedArgs& a, const double* v, int nit, bool check_last) const
    {
        if (a.timing) return;
        SolveState& s = *a.st;
        s.par_u ^= 1;
        s.par_p ^= 1;
        for (int k = 0; k < nit - 1; ++k) {
            s.cheby_calc_steps = s.cheby_calc_steps + 1;
            end_iteration(a, s, PHASE_CHEBY);  // cannot end the loop (pass_ok)
        }
        if (check_last) s.error = v[0];
        s.cheby_calc_steps = s.cheby_calc_steps + 1;
        end_iteration(a, s, PHASE_CHEBY);
    }
};

#if TEA_DIM == 2
// Two Chebyshev iterations in one pass over the 2D field (temporal blocking).  The
// iterations between two convergence checks are free of reductions, so two of them can
// share one read of u, u0, p, Kx, Ky (and mi) and one write of u and p: 7 words per cell
// for two iterations instead of fourteen.  The per-cell arithmetic is exactly that of two
// single iterations (same operations, same order), so results are bit-identical.
//
// Each warp loads a strip of 64 columns (two per lane) and marches rows through a
// shared-memory ring filled by cp.async.  Iteration 1 is computed for every loaded cell
// one row ahead of iteration 2; iteration 2 needs iteration-1 values of its x-neighbours,
// so the strip's outer lanes (0 and 31) only feed their neighbours and each warp writes
// the 60 columns of lanes 1..30 -- neighbouring strips overlap by four columns, and p is
// written to the second buffer so that no warp reads a value another warp has updated.
// Row segments overlap by one row of iteration 1 for the same reason.  At the domain's
// edges the intermediate u is reflected as the reference's halo update reflects it.
//
// A pair runs only when its first iteration is not a convergence check (which must end a
// launch) and the second stays within max_iters; otherwise the launch is one ordinary
// iteration.  Either way the decision is read from the solve state, uniformly.
constexpr int C2_RP = TEA_CHEBY2_RP;   // ring rows in flight beyond row t+1
constexpr int C2_RQ = C2_RP + 3;       // ring rows per warp: t-1 .. t+1+C2_RP
constexpr int C2_NA = 6;               // u, u0, p, mi, Kx, Ky
enum { C2_U = 0, C2_U0 = 1, C2_P = 2, C2_MI = 3, C2_KX = 4, C2_KY = 5 };

// Strips of the two-iteration kernel: 32 * VEC loaded columns, of which lanes 1..30 write
// OUT = 30 * VEC; the lane's first column is OUT * strip + VEC * lane - (VEC - 2), so that
// lane 1 of strip 0 starts at the first inner column.
template <class T>
struct Pair2Geom {
    static constexpr int VEC = RingGeom<T>::VEC;
    static constexpr int STRIP = RingGeom<T>::STRIP;
    static constexpr int OUT = 30 * VEC;
};

template <class Op>
constexpr size_t cheby2_smem_bytes()
{
    using T = typename Op::T;
    return (size_t)RWARPS * C2_RQ * C2_NA * Pair2Geom<T>::STRIP * sizeof(T) > ring_smem_bytes<Op>()
        ? (size_t)RWARPS * C2_RQ * C2_NA * Pair2Geom<T>::STRIP * sizeof(T)
        : ring_smem_bytes<Op>();
}

// NIT Chebyshev iterations in one pass over the 2D field (temporal blocking), the
// generalisation of the two-iteration pass above.  Level l (iteration l of the pass) is
// computed one row behind level l - 1: at loop step t, level l is at row t - l + 1, so
// each level reads the three rows of level l - 1 it needs from registers.  Each level loses
// one cell of its strip on each side, so a warp writes the cells of lanes FL .. 31 - FL
// (FL = ceil(NIT / VEC)), OUT = (32 - 2 FL) * VEC columns per strip, and row segments
// overlap by NIT - 1 rows.  At the domain's edges every level uses the cell's own value
// as its outside neighbour, which is what the reference's halo update after each iteration
// gives.  u and p go to the other buffers, as in the pair.  Per cell the operations and
// their order are those of NIT single iterations, so results are bit-identical.
template <class T, int NIT, int RPN>
struct PassGeom {
    static constexpr int VEC = RingGeom<T>::VEC;
    static constexpr int STRIP = RingGeom<T>::STRIP;
    static constexpr int FL = (NIT + VEC - 1) / VEC;  // first lane that writes
    static constexpr int OUT = (32 - 2 * FL) * VEC;
    static constexpr int RQ = NIT + RPN + 1;           // ring rows per warp
};

template <class Op, int NIT, int RPN>
constexpr size_t chebyN_smem_bytes()
{
    using T = typename Op::T;
    return (size_t)RWARPS * PassGeom<T, NIT, RPN>::RQ * C2_NA * PassGeom<T, NIT, RPN>::STRIP * sizeof(T);
}

template <class Op, int NIT, int RPN>
__device__ __forceinline__ void chebyN_body(const FusedArgs& a, Op& op, unsigned char* s_ring_raw)
{
    using T = typename Op::T;
    using G = PassGeom<T, NIT, RPN>;
    constexpr int VEC = G::VEC, STRIP = G::STRIP, OUT = G::OUT, FL = G::FL, RQ = G::RQ;
    T al[NIT], be[NIT];
#pragma unroll
    for (int l = 0; l < NIT; ++l) op.pass_coefs(a, l, al[l], be[l]);
    const bool checkN = op.pass_check(a, NIT);
    const T* mi = op.pair_mi(a);
    const bool precond = mi != nullptr;
    T* unew = op.unew;
    T* pnew = op.pnext;
    const Geom& g = a.g;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    T* ring = reinterpret_cast<T*>(s_ring_raw) + (size_t)warp * RQ * C2_NA * STRIP;
    const T* src[C2_NA] = {op.ucur, op.pair_rhs(a), op.pcur, mi, op.coef_x(a), op.coef_y(a)};
    DDVec<1> acc;
    acc.zero();
    const int xlast = g.X - HALO_PAD - 1;
    const int ylast = g.Y - HALO_PAD - 1;
    const int per_x = (g.nx + OUT - 1) / OUT;
    const int per_y = (g.ny + a.seg_rows - 1) / a.seg_rows;
    const long nseg = (long)per_x * per_y;
    const long gw = (long)blockIdx.x * RWARPS + warp, nw = (long)gridDim.x * RWARPS;
    const int cmax = (int)g.pitch - 2 * VEC + 2;
    const bool out_lane = lane >= FL && lane <= 31 - FL;
    const T zero = (T)0;
    for (long sgi = gw; sgi < nseg; sgi += nw) {
        const int xs = (int)(sgi % per_x), ys = (int)(sgi / per_x);
        // Lane FL of the strip starts at its first output column; lanes left of it in the
        // first strip start left of column 0 and only feed cells whose outside neighbour is
        // their own value, so they copy from c + VEC (in-row, 16-byte aligned).
        const int c = OUT * xs + VEC * (lane - FL) + HALO_PAD;
        const int cc = min(c < 0 ? c + VEC : c, cmax);
        const int j0 = HALO_PAD + a.seg_rows * ys;
        const int j1 = min(j0 + a.seg_rows, ylast + 1);
        const int a0 = max(HALO_PAD, j0 - (NIT - 1));        // first row of level 1
        const int t_last = j1 + NIT - 2;                    // level NIT reaches row j1 - 1
        const int rlast = min(t_last + 1, ylast + 1);       // last ring row
        auto slot = [&](int r) { return ring + (size_t)((r - a0 + 1) % RQ) * C2_NA * STRIP; };
        auto issue = [&](int r) {
            if (r <= rlast) {
                T* base = slot(r);
                const int urow = refl(r, g.Y);
                const int irow = min(max(r, HALO_PAD), ylast + 1);
#pragma unroll
                for (int k = 0; k < C2_NA; ++k) {
                    if (!src[k]) continue;
                    cp_async_16(base + k * STRIP + VEC * lane, src[k] + fidx(g, cc, k == C2_U ? urow : irow, 0));
                }
            }
            cp_async_commit();
        };
        // One level at row s: the operand rows (m: s-1, cv: s, n: s+1) of the level below,
        // its p at row s, and the ring row s (and s+1 for Ky).  Returns u and p of the level.
        auto level = [&](int l, int s, const T* m, const T* cv, const T* n, const T* pin, T* uo, T* po, bool last) {
            // Rows above the segment's first ring row are never needed (s is uniform in the
            // warp, so the shuffles below stay warp-uniform).
            if (s < a0 || s > ylast) return;
            const T* rs = slot(s);
            const T* rs1 = slot(s + 1);
            const T up = __shfl_up_sync(0xffffffffu, cv[VEC - 1], 1);
            const T dn = __shfl_down_sync(0xffffffffu, cv[0], 1);
            T kx[VEC + 1];
            ld_vec(rs + C2_KX * STRIP + VEC * lane, kx);
            kx[VEC] = __shfl_down_sync(0xffffffffu, kx[0], 1);
            T ky0[VEC], ky1[VEC], rhs[VEC], m0[VEC];
            ld_vec(rs + C2_KY * STRIP + VEC * lane, ky0);
            ld_vec(rs1 + C2_KY * STRIP + VEC * lane, ky1);
            ld_vec(rs + C2_U0 * STRIP + VEC * lane, rhs);
            if (precond) ld_vec(rs + C2_MI * STRIP + VEC * lane, m0);
#pragma unroll
            for (int q = 0; q < VEC; ++q) {
                NbT<T> nb;
                nb.zm = nb.zp = zero;
                nb.c = cv[q];
                nb.xm = c + q == HALO_PAD ? cv[q] : (q == 0 ? up : cv[q > 0 ? q - 1 : 0]);
                nb.xp = c + q == xlast ? cv[q] : (q == VEC - 1 ? dn : cv[q < VEC - 1 ? q + 1 : q]);
                nb.ym = s == HALO_PAD ? cv[q] : m[q];
                nb.yp = s == ylast ? cv[q] : n[q];
                const T w = smvp_k(nb, kx[q], kx[q + 1], ky0[q], ky1[q], zero, zero);
                const T r = rhs[q] - w;
                po[q] = al[l] * pin[q] + be[l] * (precond ? m0[q] * r : r);
                uo[q] = cv[q] + po[q];
                if (last && checkN && out_lane && c + q <= xlast) dd_add(acc.v[0], (double)r * (double)r);
            }
        };
        // Rows a0 - 1 .. a0 + RPN + 1 first; each step then issues the next new row, so row
        // t + 1 has exactly RPN groups after it at the top of step t.
        for (int r = a0 - 1; r <= a0 + RPN + 1; ++r) issue(r);
        cp_async_wait<RPN + 1>();
        __syncwarp();
        T um[VEC], uc[VEC];
        ld_vec(slot(a0 - 1) + C2_U * STRIP + VEC * lane, um);
        ld_vec(slot(a0) + C2_U * STRIP + VEC * lane, uc);
        // Level L (iteration L + 1) keeps its u at rows s - 1 (M) and s (C) and its p at row
        // s (P), where s is the row it reached at the previous step.
        T M[NIT][VEC], C[NIT][VEC], P[NIT][VEC];
#pragma unroll
        for (int l = 0; l < NIT; ++l)
#pragma unroll
            for (int q = 0; q < VEC; ++q) M[l][q] = C[l][q] = P[l][q] = zero;
        for (int t = a0; t <= t_last; ++t) {
            cp_async_wait<RPN>();
            __syncwarp();
            T un[VEC], p0[VEC];
            ld_vec(slot(t + 1) + C2_U * STRIP + VEC * lane, un);
            ld_vec(slot(t) + C2_P * STRIP + VEC * lane, p0);
            T N[NIT][VEC], PN[NIT][VEC];
#pragma unroll
            for (int l = 0; l < NIT; ++l)
#pragma unroll
                for (int q = 0; q < VEC; ++q) N[l][q] = PN[l][q] = zero;
            level(0, t, um, uc, un, p0, N[0], PN[0], NIT == 1 && t >= j0);
#pragma unroll
            for (int l = 1; l < NIT; ++l) {
                const int s = t - l;
                level(l, s, M[l - 1], C[l - 1], N[l - 1], P[l - 1], N[l], PN[l], l == NIT - 1 && s >= j0);
            }
            const int sl = t - NIT + 1;  // the row the last level reached
            if (sl >= j0 && sl <= ylast && out_lane) {
                const long i = fidx(g, c, sl, 0);
                if (c + VEC - 1 <= xlast) {
                    st_vec(unew + i, N[NIT - 1]);
                    st_vec(pnew + i, PN[NIT - 1]);
                } else {
#pragma unroll
                    for (int q = 0; q < VEC; ++q) {
                        if (c + q <= xlast) {
                            unew[i + q] = N[NIT - 1][q];
                            pnew[i + q] = PN[NIT - 1][q];
                        }
                    }
                }
            }
#pragma unroll
            for (int l = 0; l < NIT; ++l)
#pragma unroll
                for (int q = 0; q < VEC; ++q) {
                    M[l][q] = C[l][q];
                    C[l][q] = N[l][q];
                    P[l][q] = PN[l][q];
                }
#pragma unroll
            for (int q = 0; q < VEC; ++q) {
                um[q] = uc[q];
                uc[q] = un[q];
            }
            __syncwarp();
            issue(t + RPN + 2);  // into the slot of row t - NIT + 1, which no lane reads any more
        }
        cp_async_wait<0>();
        __syncwarp();
    }
    grid_reduce_then<1>(acc, a.red, [&](const double* v) { op.pass_control(a, v, NIT, checkN); });
}

// NIT Chebyshev iterations in one pass with the levels skewed by two rows: at loop step t,
// level l (iteration l of the pass) computes row t - 2l.  Level l at row s reads level
// l - 1 at rows s - 1, s, s + 1, which level l - 1 produced at steps t - 3, t - 2, t - 1, so
// no level waits on another within a step and a lane's NIT * VEC cell updates of a step are
// independent chains (with one row of skew, as in chebyN_body, each level waits for the
// one below, and the pass was bound by that dependency latency).  The strips, the
// overlap of strips and segments, the edge handling and the per-cell operations are those of
// chebyN_body, so the results are the same bits.
//
// Rings, per warp: the coefficient rows (u0, Kx, Ky and, when preconditioned, mi) of rows
// t - 2(NIT - 1) .. t + 1 + RPN, which every level reads, and the operand rows (u, p) of
// rows t - 1 .. t + 1 + RPN, which only level 0 reads.  Each level keeps its last three u
// rows and two p rows in registers for the level above.  Away from the domain's edges
// (warp-uniform per level and row) a cell takes its neighbours without the edge selects.
template <class T, int NIT, int RPN>
struct SkewGeom {
    static constexpr int VEC = RingGeom<T>::VEC;
    static constexpr int STRIP = RingGeom<T>::STRIP;
    static constexpr int FL = (NIT + VEC - 1) / VEC;  // first lane that writes
    static constexpr int OUT = (32 - 2 * FL) * VEC;
    static constexpr int RQC = 2 * (NIT - 1) + RPN + 2;  // coefficient ring rows per warp
    static constexpr int RQO = RPN + 3;                  // operand ring rows per warp
};
enum { S_U0 = 0, S_KX = 1, S_KY = 2, S_MI = 3 };  // coefficient arrays of a ring row

template <class T, int NIT, int RPN>
constexpr size_t chebyS_warp_bytes(bool precond)
{
    using G = SkewGeom<T, NIT, RPN>;
    return (size_t)((precond ? 4 : 3) * G::RQC + 2 * G::RQO) * G::STRIP * sizeof(T);
}

// PRE: the preconditioned form (mi staged and applied); the caller picks it from op.pair_mi.
template <class Op, int NIT, int RPN, bool PRE>
__device__ __forceinline__ void chebyS_body(const FusedArgs& a, Op& op, unsigned char* s_ring_raw)
{
    using T = typename Op::T;
    using G = SkewGeom<T, NIT, RPN>;
    constexpr int VEC = G::VEC, STRIP = G::STRIP, OUT = G::OUT, FL = G::FL, RQC = G::RQC, RQO = G::RQO;
    // The pass's coefficients in shared memory (two loads per level and row instead of 2 NIT
    // registers held through the loop).
    __shared__ T s_coef[2 * NIT];
    if (threadIdx.x < NIT) op.pass_coefs(a, threadIdx.x, s_coef[threadIdx.x], s_coef[NIT + threadIdx.x]);
    __syncthreads();
    const bool checkN = op.pass_check(a, NIT);
    const T* mi = op.pair_mi(a);
    constexpr int nc = PRE ? 4 : 3;
    T* unew = op.unew;
    T* pnew = op.pnext;
    const Geom& g = a.g;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    T* cring = reinterpret_cast<T*>(s_ring_raw) + (size_t)warp * (nc * RQC + 2 * RQO) * STRIP;
    T* oring = cring + (size_t)nc * RQC * STRIP;
    const T* csrc[4] = {op.pair_rhs(a), op.coef_x(a), op.coef_y(a), mi};
    const T* usrc = op.ucur;
    const T* psrc = op.pcur;
    DDVec<1> acc;
    acc.zero();
    const int xlast = g.X - HALO_PAD - 1;
    const int ylast = g.Y - HALO_PAD - 1;
    const int per_x = (g.nx + OUT - 1) / OUT;
    const int per_y = (g.ny + a.seg_rows - 1) / a.seg_rows;
    const long nseg = (long)per_x * per_y;
    const long gw = (long)blockIdx.x * RWARPS + warp, nw = (long)gridDim.x * RWARPS;
    const int cmax = (int)g.pitch - 2 * VEC + 2;
    const bool out_lane = lane >= FL && lane <= 31 - FL;
    const T zero = (T)0;
    auto wrap_c = [](int x) { return x >= RQC ? x - RQC : x; };  // x < 2 RQC
    auto wrap_o = [](int x) { return x >= RQO ? x - RQO : x; };  // x < 2 RQO
    for (long sgi = gw; sgi < nseg; sgi += nw) {
        const int xs = (int)(sgi % per_x), ys = (int)(sgi / per_x);
        const int c = OUT * xs + VEC * (lane - FL) + HALO_PAD;
        const int cc = min(c < 0 ? c + VEC : c, cmax);
        // Does the strip hold the first or the last inner column (edge selects needed)?
        const bool xedge = __any_sync(0xffffffffu, c == HALO_PAD || (c <= xlast && xlast < c + VEC));
        const int j0 = HALO_PAD + a.seg_rows * ys;
        const int j1 = min(j0 + a.seg_rows, ylast + 1);
        const int a0 = max(HALO_PAD, j0 - (NIT - 1));        // first row of level 1
        const int t_last = j1 - 1 + 2 * (NIT - 1);          // the last level reaches row j1 - 1
        const int rlast = min(j1 + NIT - 1, ylast + 1);     // last ring row (level 0 needs rows to j1 + NIT - 2)
        // Ring index of row r is (r - a0 + 1) mod RQC (coefficients) and mod RQO (operands).
        auto issue = [&](int r, int ci, int oi) {
            if (r <= rlast) {
                T* cb = cring + (size_t)ci * nc * STRIP + VEC * lane;
                T* ob = oring + (size_t)oi * 2 * STRIP + VEC * lane;
                const int urow = refl(r, g.Y);
                const int irow = min(max(r, HALO_PAD), ylast + 1);
#pragma unroll
                for (int k = 0; k < nc; ++k) cp_async_16(cb + k * STRIP, csrc[k] + fidx(g, cc, irow, 0));
                cp_async_16(ob, usrc + fidx(g, cc, urow, 0));
                cp_async_16(ob + STRIP, psrc + fidx(g, cc, irow, 0));
            }
            cp_async_commit();
        };
        // Level l at row s (ring index ci): the operand rows m (s - 1), cv (s), n (s + 1) and
        // p of the level below; u, p and r of the level into uo, po, ro.  Every level runs at
        // every step, also at rows outside its useful range (above the segment's first ring
        // row, past the rows the last level needs, past the domain), whose values reach no
        // stored or summed cell: the step then has no branch, and the levels' independent
        // chains interleave.  EDGE (warp-uniform): some cell of the step sits at a domain
        // edge, where the neighbour is the cell's own value.
        auto level = [&](auto edge_tag, int l, int s, int ci, const T* m, const T* cv, const T* n, const T* pin,
                         T* uo, T* po, T* ro) {
            constexpr bool EDGE = decltype(edge_tag)::value;
            const T* rs = cring + (size_t)ci * nc * STRIP + VEC * lane;
            const T* rs1 = cring + (size_t)wrap_c(ci + 1) * nc * STRIP + VEC * lane;
            const T up = __shfl_up_sync(0xffffffffu, cv[VEC - 1], 1);
            const T dn = __shfl_down_sync(0xffffffffu, cv[0], 1);
            T kx[VEC + 1];
            ld_vec(rs + S_KX * STRIP, kx);
            kx[VEC] = rs[S_KX * STRIP + VEC];  // the next lane's first Kx (lane 31: never used)
            T ky0[VEC], ky1[VEC], rhs[VEC], m0[PRE ? VEC : 1];
            ld_vec(rs + S_KY * STRIP, ky0);
            ld_vec(rs1 + S_KY * STRIP, ky1);
            ld_vec(rs + S_U0 * STRIP, rhs);
            if constexpr (PRE) ld_vec(rs + S_MI * STRIP, m0);
            else (void)m0;
#pragma unroll
            for (int q = 0; q < VEC; ++q) {
                NbT<T> nb;
                nb.zm = nb.zp = zero;
                nb.c = cv[q];
                if constexpr (EDGE) {
                    nb.xm = c + q == HALO_PAD ? cv[q] : (q == 0 ? up : cv[q > 0 ? q - 1 : 0]);
                    nb.xp = c + q == xlast ? cv[q] : (q == VEC - 1 ? dn : cv[q < VEC - 1 ? q + 1 : q]);
                    nb.ym = s == HALO_PAD ? cv[q] : m[q];
                    nb.yp = s == ylast ? cv[q] : n[q];
                } else {
                    nb.xm = q == 0 ? up : cv[q > 0 ? q - 1 : 0];
                    nb.xp = q == VEC - 1 ? dn : cv[q < VEC - 1 ? q + 1 : q];
                    nb.ym = m[q];
                    nb.yp = n[q];
                }
                const T w = smvp_k(nb, kx[q], kx[q + 1], ky0[q], ky1[q], zero, zero);
                const T r = rhs[q] - w;
                T pr;
                if constexpr (PRE) pr = s_coef[l] * pin[q] + s_coef[NIT + l] * (m0[q] * r);
                else pr = s_coef[l] * pin[q] + s_coef[NIT + l] * r;
                po[q] = pr;
                uo[q] = cv[q] + pr;
                ro[q] = r;
            }
        };
        // Rows a0 - 1 .. a0 + RPN + 1 first; each step then issues the next new row, so row
        // t + 1 has exactly RPN groups after it at the top of step t.
        for (int r = a0 - 1; r <= a0 + RPN + 1; ++r) issue(r, (r - a0 + 1) % RQC, (r - a0 + 1) % RQO);
        cp_async_wait<RPN + 1>();
        __syncwarp();
        // Register windows of three rows, indexed by the step's phase k = (t - a0) mod 3 so
        // that the loop, unrolled by three, moves no registers: U0 holds level 0's operand
        // rows (row r at (r - a0 + 1) mod 3: rows t - 1, t, t + 1 at k, k + 1, k + 2), and
        // H[l] / PH[l] the u / p rows level l < NIT - 1 produced at the last three steps
        // (step s at (s - a0) mod 3: steps t - 3, t - 2, t - 1 at k, k + 1, k + 2).
        T U0[3][VEC], H[NIT - 1][3][VEC], PH[NIT - 1][3][VEC];
        ld_vec(oring + VEC * lane, U0[0]);                                   // row a0 - 1
        ld_vec(oring + (size_t)(1 % RQO) * 2 * STRIP + VEC * lane, U0[1]);  // row a0
#pragma unroll
        for (int l = 0; l < NIT - 1; ++l)
#pragma unroll
            for (int h = 0; h < 3; ++h)
#pragma unroll
                for (int q = 0; q < VEC; ++q) H[l][h][q] = PH[l][h][q] = zero;
        int ct = 1 % RQC, ot = 1 % RQO;  // ring indices of row t
        // One step at row t of phase K.
        auto step = [&](auto phase_tag, int t) {
            constexpr int K = decltype(phase_tag)::value;
            constexpr int K1 = (K + 1) % 3, K2 = (K + 2) % 3;
            cp_async_wait<RPN>();
            __syncwarp();
            T p0[VEC];
            ld_vec(oring + (size_t)wrap_o(ot + 1) * 2 * STRIP + VEC * lane, U0[K2]);  // row t + 1
            ld_vec(oring + (size_t)ot * 2 * STRIP + STRIP + VEC * lane, p0);
            T NU[NIT][VEC], NP[NIT][VEC], RR[VEC];
            auto levels = [&](auto edge_tag) {
                level(edge_tag, 0, t, ct, U0[K], U0[K1], U0[K2], p0, NU[0], NP[0], RR);
#pragma unroll
                for (int l = 1; l < NIT; ++l)
                    level(edge_tag, l, t - 2 * l, wrap_c(ct + RQC - 2 * l), H[l - 1][K], H[l - 1][K1], H[l - 1][K2],
                          PH[l - 1][K1], NU[l], NP[l], RR);
            };
            bool yedge = false;
#pragma unroll
            for (int l = 0; l < NIT; ++l) yedge = yedge || t - 2 * l == HALO_PAD || t - 2 * l == ylast;
            if (xedge || yedge) levels(std::true_type{});
            else levels(std::false_type{});
            // The last level's sum r.r on a convergence-check pass, over the cells it writes
            // (adding 0.0 leaves a double-double sum unchanged).
            const int sl = t - 2 * (NIT - 1);  // the row the last level reached
            if (checkN && sl >= j0 && sl < j1) {
#pragma unroll
                for (int q = 0; q < VEC; ++q)
                    dd_add(acc.v[0], out_lane && c + q <= xlast ? (double)RR[q] * (double)RR[q] : 0.0);
            }
            if (sl >= j0 && sl < j1 && out_lane) {
                const long i = fidx(g, c, sl, 0);
                if (c + VEC - 1 <= xlast) {
                    st_vec(unew + i, NU[NIT - 1]);
                    st_vec(pnew + i, NP[NIT - 1]);
                } else {
#pragma unroll
                    for (int q = 0; q < VEC; ++q) {
                        if (c + q <= xlast) {
                            unew[i + q] = NU[NIT - 1][q];
                            pnew[i + q] = NP[NIT - 1][q];
                        }
                    }
                }
            }
            // Step t's rows replace those of step t - 3 (slot K).
#pragma unroll
            for (int l = 0; l < NIT - 1; ++l)
#pragma unroll
                for (int q = 0; q < VEC; ++q) {
                    H[l][K][q] = NU[l][q];
                    PH[l][K][q] = NP[l][q];
                }
            __syncwarp();
            // Row t + RPN + 2 goes into the coefficient slot of row t - 2(NIT - 1) and the
            // operand slot of row t - 1, which no lane reads any more.
            issue(t + RPN + 2, wrap_c(ct + RPN + 2), wrap_o(ot + RPN + 2));
            ct = wrap_c(ct + 1);
            ot = wrap_o(ot + 1);
        };
        using P0 = std::integral_constant<int, 0>;
        using P1 = std::integral_constant<int, 1>;
        using P2 = std::integral_constant<int, 2>;
        int t = a0;
        for (; t + 2 <= t_last; t += 3) {
            step(P0{}, t);
            step(P1{}, t + 1);
            step(P2{}, t + 2);
        }
        if (t <= t_last) step(P0{}, t);
        if (t + 1 <= t_last) step(P1{}, t + 1);
        cp_async_wait<0>();
        __syncwarp();
    }
    grid_reduce_then<1>(acc, a.red, [&](const double* v) { op.pass_control(a, v, NIT, checkN); });
}

// Op: OpCheby (FP64, the reference's iteration) or OpCheby32 (the FP32 inner solve).  Two
// iterations when the state allows (pass_ok), else one.
template <class Op>
__global__ void __launch_bounds__(RWARPS * 32) k_cheby2_ring2d(FusedArgs a)
{
    extern __shared__ __align__(16) unsigned char s_ring_raw[];
    Op op;
    op.begin(a);
    if (op.pass_ok(a, 2)) chebyN_body<Op, 2, C2_RP>(a, op, s_ring_raw);
    else ring2d_body(a, op, s_ring_raw);
}

// Four iterations (skewed levels) when the state allows, else two, else one.  The shared
// memory a launch needs depends on whether mi is staged (the preconditioned FP64 solve).
constexpr int C4_RP = 1;  // ring rows in flight beyond row t+1 in the four-iteration pass
template <class Op>
constexpr size_t cheby4_smem_bytes(bool precond)
{
    using T = typename Op::T;
    const size_t quad = (size_t)RWARPS * chebyS_warp_bytes<T, 4, C4_RP>(precond);
    return quad > cheby2_smem_bytes<Op>() ? quad : cheby2_smem_bytes<Op>();
}
template <class Op>
__global__ void __launch_bounds__(RWARPS * 32, 3) k_cheby4_ring2d(FusedArgs a)
{
    extern __shared__ __align__(16) unsigned char s_ring_raw[];
    Op op;
    op.begin(a);
    if (op.pass_ok(a, 4)) {
        if (op.pair_mi(a)) chebyS_body<Op, 4, C4_RP, true>(a, op, s_ring_raw);
        else chebyS_body<Op, 4, C4_RP, false>(a, op, s_ring_raw);
    } else if (op.pass_ok(a, 2)) {
        chebyN_body<Op, 2, C2_RP>(a, op, s_ring_raw);
    } else {
        ring2d_body(a, op, s_ring_raw);
    }
}

// Two PPCG inner steps in one pass over the 2D field (temporal blocking), the 2D form of
// k_ppcg2_ring3d on the strips and row rings of k_cheby2_ring2d: step k is computed for
// every loaded cell one row ahead of step k+1, the strips' outer lanes and a segment's
// first row only feed their neighbours, and at the domain's edges step k's sd is
// reflected as the reference's halo update reflects it.  Per cell the operations and their
// order are those of two single steps, so results are bit-identical.  r moves between r
// and w and sd between its two buffers, and a pair may hold the last, reducing step, all as
// in 3D; u is read and written only at the cells a warp writes.
enum { P2_SD = 0, P2_R = 1, P2_U = 2, P2_MI = 3, P2_KX = 4, P2_KY = 5 };

template <class P>
__global__ void __launch_bounds__(RWARPS * 32) k_ppcg2_ring2d(FusedArgs a)
{
    using T = typename P::T;
    constexpr int VEC = Pair2Geom<T>::VEC, STRIP = Pair2Geom<T>::STRIP, OUT = Pair2Geom<T>::OUT;
    extern __shared__ __align__(16) unsigned char s_ring_raw[];
    const int k = a.step;
    const int m = (k + 1) >> 1;
    const T* __restrict__ sdk = P::sd(a, (m - 1) & 1);
    T* __restrict__ sdo = P::sd(a, m & 1);
    const T* __restrict__ rin = ((m - 1 + a.r_in_w) & 1) ? P::w(a) : P::r(a);
    T* __restrict__ rout = ((m + a.r_in_w) & 1) ? P::w(a) : P::r(a);
    T* __restrict__ U = P::u(a);
    const T* __restrict__ mi = P::mi(a);
    const bool precond = mi != nullptr;
    const bool last = k + 1 == a.st->inner_steps;  // step k+1 ends the outer iteration
    DDVec<1> acc;
    acc.zero();
    const T al1 = (T)a.ch_alphas[k - 1], be1 = (T)a.ch_betas[k - 1];
    const T al2 = (T)a.ch_alphas[k], be2 = (T)a.ch_betas[k];
    const Geom& g = a.g;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    T* ring = reinterpret_cast<T*>(s_ring_raw) + (size_t)warp * C2_RQ * C2_NA * STRIP;
    const T* src[C2_NA] = {sdk, rin, U, mi, P::kx(a), P::ky(a)};
    const int xlast = g.X - HALO_PAD - 1;
    const int ylast = g.Y - HALO_PAD - 1;
    const int per_x = (g.nx + OUT - 1) / OUT;
    const int per_y = (g.ny + a.seg_rows - 1) / a.seg_rows;
    const long nseg = (long)per_x * per_y;
    const long gw = (long)blockIdx.x * RWARPS + warp, nw = (long)gridDim.x * RWARPS;
    const int cmax = (int)g.pitch - 2 * VEC + 2;
    const bool out_lane = lane >= 1 && lane <= 30;
    for (long sgi = gw; sgi < nseg; sgi += nw) {
        const int xs = (int)(sgi % per_x), ys = (int)(sgi / per_x);
        const int c = OUT * xs + VEC * lane - (VEC - 2);  // the lane's first column (>= -2: the lead pad)
        const int cc = min(c, cmax);
        const int j0 = HALO_PAD + a.seg_rows * ys;
        const int j1 = min(j0 + a.seg_rows, ylast + 1);
        const int a0 = j0 == HALO_PAD ? HALO_PAD : j0 - 1;  // first row of step k
        const int rlast = min(j1 + 1, ylast + 1);             // last ring row
        auto slot = [&](int r) { return ring + (size_t)((r - a0 + 1) % C2_RQ) * C2_NA * STRIP; };
        auto issue = [&](int r) {
            if (r <= rlast) {
                T* base = slot(r);
                const int srow = refl(r, g.Y);
                const int irow = min(max(r, HALO_PAD), ylast + 1);
#pragma unroll
                for (int q = 0; q < C2_NA; ++q) {
                    if (!src[q]) continue;
                    if (q == P2_U && !(out_lane && r >= j0 && r < j1)) continue;  // u: written cells only
                    cp_async_16(base + q * STRIP + VEC * lane, src[q] + fidx(g, cc, q == P2_SD ? srow : irow, 0));
                }
            }
            cp_async_commit();
        };
        for (int r = a0 - 1; r <= a0 + C2_RP + 1; ++r) issue(r);
        cp_async_wait<C2_RP + 1>();
        __syncwarp();
        // sd at rows t-1 (um) and t (uc); step k's sd at rows t-2 (vm) and t-1 (vc), its r
        // and u at row t-1 (r1c, u1c).
        T um[VEC], uc[VEC], vm[VEC], vc[VEC], r1c[VEC], u1c[VEC];
        ld_vec(slot(a0 - 1) + P2_SD * STRIP + VEC * lane, um);
        ld_vec(slot(a0) + P2_SD * STRIP + VEC * lane, uc);
#pragma unroll
        for (int q = 0; q < VEC; ++q) vm[q] = vc[q] = r1c[q] = u1c[q] = (T)0;
        for (int t = a0; t <= j1; ++t) {
            cp_async_wait<C2_RP>();
            __syncwarp();
            const T* rp = slot(t - 1);
            const T* rc = slot(t);
            const T* rn = slot(t + 1);
            T un[VEC];
            ld_vec(rn + P2_SD * STRIP + VEC * lane, un);
            // Step k at row t.
            T v[VEC], r1v[VEC], u1v[VEC];
            if (t <= ylast) {
                T kx[VEC + 1], ky0[VEC], ky1[VEC], rr[VEC], uu[VEC], m0[VEC];
                ld_vec(rc + P2_KX * STRIP + VEC * lane, kx);
                kx[VEC] = __shfl_down_sync(0xffffffffu, kx[0], 1);
                ld_vec(rc + P2_KY * STRIP + VEC * lane, ky0);
                ld_vec(rn + P2_KY * STRIP + VEC * lane, ky1);
                ld_vec(rc + P2_R * STRIP + VEC * lane, rr);
                ld_vec(rc + P2_U * STRIP + VEC * lane, uu);
                if (precond) ld_vec(rc + P2_MI * STRIP + VEC * lane, m0);
                const T up = __shfl_up_sync(0xffffffffu, uc[VEC - 1], 1);
                const T dn = __shfl_down_sync(0xffffffffu, uc[0], 1);
#pragma unroll
                for (int q = 0; q < VEC; ++q) {
                    NbT<T> nb;
                    nb.zm = nb.zp = (T)0;
                    nb.c = uc[q];
                    nb.xm = c + q == HALO_PAD ? uc[q] : (q == 0 ? up : uc[q > 0 ? q - 1 : 0]);
                    nb.xp = c + q == xlast ? uc[q] : (q == VEC - 1 ? dn : uc[q < VEC - 1 ? q + 1 : q]);
                    nb.ym = um[q];
                    nb.yp = un[q];
                    const T s = smvp_k(nb, kx[q], kx[q + 1], ky0[q], ky1[q], (T)0, (T)0);
                    const T r = rr[q] - s;
                    r1v[q] = r;
                    u1v[q] = uu[q] + uc[q];
                    v[q] = al1 * uc[q] + be1 * (precond ? m0[q] * r : r);
                }
            } else {
                // Row ylast + 1 is the halo: the reflection of row ylast.
#pragma unroll
                for (int q = 0; q < VEC; ++q) {
                    v[q] = vc[q];
                    r1v[q] = u1v[q] = (T)0;
                }
            }
            if (t == HALO_PAD) {
                // Row 1 is the halo: the reflection of row 2.
#pragma unroll
                for (int q = 0; q < VEC; ++q) vc[q] = v[q];
            }
            // Step k+1 at row s = t - 1.
            const int srow = t - 1;
            if (srow >= j0) {
                T kx[VEC + 1], ky0[VEC], ky1[VEC], m0[VEC], r2[VEC], u2[VEC], d2[VEC];
                ld_vec(rp + P2_KX * STRIP + VEC * lane, kx);
                kx[VEC] = __shfl_down_sync(0xffffffffu, kx[0], 1);
                ld_vec(rp + P2_KY * STRIP + VEC * lane, ky0);
                ld_vec(rc + P2_KY * STRIP + VEC * lane, ky1);
                if (precond) ld_vec(rp + P2_MI * STRIP + VEC * lane, m0);
                const T up = __shfl_up_sync(0xffffffffu, vc[VEC - 1], 1);
                const T dn = __shfl_down_sync(0xffffffffu, vc[0], 1);
                const long i = fidx(g, c, srow, 0);
#pragma unroll
                for (int q = 0; q < VEC; ++q) {
                    NbT<T> nb;
                    nb.zm = nb.zp = (T)0;
                    nb.c = vc[q];
                    nb.xm = c + q == HALO_PAD ? vc[q] : (q == 0 ? up : vc[q > 0 ? q - 1 : 0]);
                    nb.xp = c + q == xlast ? vc[q] : (q == VEC - 1 ? dn : vc[q < VEC - 1 ? q + 1 : q]);
                    nb.ym = vm[q];
                    nb.yp = v[q];
                    const T s = smvp_k(nb, kx[q], kx[q + 1], ky0[q], ky1[q], (T)0, (T)0);
                    const T r = r1c[q] - s;
                    r2[q] = r;
                    u2[q] = u1c[q] + vc[q];
                    d2[q] = al2 * vc[q] + be2 * (precond ? m0[q] * r : r);
                    if (last && out_lane && c + q <= xlast) dd_add(acc.v[0], (double)r * (double)r);
                }
                if (out_lane && c + VEC - 1 <= xlast) {
                    st_vec(rout + i, r2);
                    st_vec(U + i, u2);
                    st_vec(sdo + i, d2);
                } else if (out_lane) {
#pragma unroll
                    for (int q = 0; q < VEC; ++q) {
                        if (c + q <= xlast) {
                            rout[i + q] = r2[q];
                            U[i + q] = u2[q];
                            sdo[i + q] = d2[q];
                        }
                    }
                }
            }
#pragma unroll
            for (int q = 0; q < VEC; ++q) {
                vm[q] = vc[q];
                vc[q] = v[q];
                r1c[q] = r1v[q];
                u1c[q] = u1v[q];
                um[q] = uc[q];
                uc[q] = un[q];
            }
            __syncwarp();
            issue(t + C2_RP + 2);  // into the slot of row t - 1, which no lane reads any more
        }
        cp_async_wait<0>();
        __syncwarp();
    }
    // The last inner step's sum r.r and the end of the outer iteration.
    if (last) grid_reduce_then<1>(acc, a.red, [&](const double* v) { P::control(a, v); });
}
#endif

// ------------------------------------------------------------------ Jacobi

// JacobiCopyU + JacobiSolve (tealeaf_2d/ext_jacobi_kernel.hpp:66-117) with u
// double-buffered instead of copied: u_new from the staged u_old, error = sum|u_new-u_old|.
struct OpJacobi {
    static constexpr bool kReduce = true;
    using T = double;
    static constexpr int NV = 1;
    __device__ const double* coef_x(const FusedArgs& a) const { return a.kx; }
    __device__ const double* coef_y(const FusedArgs& a) const { return a.ky; }
    __device__ const double* coef_z(const FusedArgs& a) const { return a.kz; }
    const double* ucur;
    double* unew;
    __device__ bool skip(const FusedArgs&) { return false; }
    __device__ void begin(const FusedArgs& a)
    {
        const SolveState& s = *a.st;
        ucur = a.u[s.par_u];
        unew = a.u[s.par_u ^ 1];
    }
    struct Raw {
        double u;
    };
    struct In {
        double u0;
    };
    __device__ Raw load_raw(const FusedArgs&, long i) const
    {
        Raw r;
        r.u = ucur[i];
        return r;
    }
    __device__ double stage_raw(const Raw& r) const { return r.u; }
    __device__ In load_in(const FusedArgs& a, long i) const
    {
        In in;
        in.u0 = a.u0[i];
        return in;
    }
    static constexpr int NR = 1, NI = 1;
    __device__ const double* raw_ptr(const FusedArgs& a, int) const { (void)a; return ucur; }
    __device__ const double* in_ptr(const FusedArgs& a, int) const { return a.u0; }
    __device__ Raw raw_from(const double* v) const
    {
        Raw r;
        r.u = v[0];
        return r;
    }
    __device__ In in_from(const double* v) const
    {
        In in;
        in.u0 = v[0];
        return in;
    }
    __device__ void interior_k(const FusedArgs&, long i, const Nb& nb, const Raw&, const In& in, double kx0,
                               double kx1, double ky0, double ky1, double kz0, double kz1, DDVec<1>& acc) const
    {
        const double un = jacobi_k(in.u0, nb, kx0, kx1, ky0, ky1, kz0, kz1);
        unew[i] = un;
        dd_add(acc.v[0], fabs(un - nb.c));
    }
    __device__ void control(const FusedArgs& a, const double* v)
    {
        const double err = v[0];
        if (a.timing) return;
        SolveState& s = *a.st;
        s.par_u ^= 1;
        s.error = err;
        if (s.n % 50 == 0) {
            s.resid_pending = 1;  // tealeaf_2d/tea_solve.f90:458-482: true residual this iteration
        } else {
            end_iteration(a, s, PHASE_JACOBI);
        }
    }
};

// CalculateResidual + Calculate2Norm(r) (tealeaf_2d/ext_solver_methods.hpp:38-92) on the
// Jacobi iterations that check the true residual; a no-op launch otherwise.
struct OpJacobiResidual {
    static constexpr bool kReduce = true;
    using T = double;
    static constexpr int NV = 1;
    __device__ const double* coef_x(const FusedArgs& a) const { return a.kx; }
    __device__ const double* coef_y(const FusedArgs& a) const { return a.ky; }
    __device__ const double* coef_z(const FusedArgs& a) const { return a.kz; }
    const double* ucur;
    __device__ bool skip(const FusedArgs& a) { return a.st->resid_pending == 0; }
    __device__ void begin(const FusedArgs& a) { ucur = a.u[a.st->par_u]; }
    struct Raw {
        double u;
    };
    struct In {
        double u0;
    };
    __device__ Raw load_raw(const FusedArgs&, long i) const
    {
        Raw r;
        r.u = ucur[i];
        return r;
    }
    __device__ double stage_raw(const Raw& r) const { return r.u; }
    __device__ In load_in(const FusedArgs& a, long i) const
    {
        In in;
        in.u0 = a.u0[i];
        return in;
    }
    static constexpr int NR = 1, NI = 1;
    __device__ const double* raw_ptr(const FusedArgs& a, int) const { (void)a; return ucur; }
    __device__ const double* in_ptr(const FusedArgs& a, int) const { return a.u0; }
    __device__ Raw raw_from(const double* v) const
    {
        Raw r;
        r.u = v[0];
        return r;
    }
    __device__ In in_from(const double* v) const
    {
        In in;
        in.u0 = v[0];
        return in;
    }
    __device__ void interior_k(const FusedArgs& a, long i, const Nb& nb, const Raw&, const In& in, double kx0,
                               double kx1, double ky0, double ky1, double kz0, double kz1, DDVec<1>& acc) const
    {
        const double s = smvp_k(nb, kx0, kx1, ky0, ky1, kz0, kz1);
        const double r = in.u0 - s;
        a.r[i] = r;
        dd_add(acc.v[0], r * r);
    }
    __device__ void control(const FusedArgs& a, const double* v)
    {
        const double rr = v[0];
        if (a.timing) return;
        SolveState& s = *a.st;
        s.error = rr;
        s.resid_pending = 0;
        end_iteration(a, s, PHASE_JACOBI);
    }
};

// ------------------------------------------------------------------ FP32 defect correction
//
// The precision form: FP64 keeps the outer residual r = b - A u, the update of u, the sums
// that decide convergence and the field summary; the inner correction solve A d = r runs
// CG with FP32 storage and arithmetic (its dot products accumulate the FP32 products in
// double-double), halving the bytes of every inner iteration.

// Kx/Ky/Kz rounded to FP32 once per solve (padded arrays, pointwise).
__global__ void __launch_bounds__(256) k_coef_to_fp32(FusedArgs a)
{
    const Geom& g = a.g;
    const long n = (long)g.page * g.Z;
    const long base = -(long)kLeadPad;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n + kLeadPad; t += (long)gridDim.x * blockDim.x) {
        const long i = base + t;
        a.kx32[i] = (float)a.kx[i];
        a.ky32[i] = (float)a.ky[i];
        if (DIM == 3) a.kz32[i] = (float)a.kz[i];
    }
}

// Outer residual in FP64 (CalculateResidual + Calculate2Norm), seeding the FP32 inner
// solve: r32 = fl32(r), and for CG p32 = r32, d32 = 0, for Chebyshev its first step
// p32 = d32 = r32 / theta; sums: r.r (FP64, decides outer convergence) and r32.r32 (the
// inner rro / reference norm).
struct OpOuterResid {
    static constexpr bool kReduce = true;
    using T = double;
    static constexpr int NV = 2;
    __device__ const double* coef_x(const FusedArgs& a) const { return a.kx; }
    __device__ const double* coef_y(const FusedArgs& a) const { return a.ky; }
    __device__ const double* coef_z(const FusedArgs& a) const { return a.kz; }
    struct Raw {
        double u;
    };
    struct In {
        double u0;
    };
    int cheby;      // seed the inner Chebyshev solve (else the inner CG)
    float theta32;  // its first step d = p = r / theta
    __device__ bool skip(const FusedArgs&) { return false; }
    __device__ void begin(const FusedArgs& a)
    {
        cheby = a.st->inner_cheby == 1;
        theta32 = (float)a.st->theta;
    }
    __device__ Raw load_raw(const FusedArgs& a, long i) const
    {
        Raw r;
        r.u = a.u[0][i];
        return r;
    }
    __device__ double stage_raw(const Raw& r) const { return r.u; }
    __device__ In load_in(const FusedArgs& a, long i) const
    {
        In in;
        in.u0 = a.u0[i];
        return in;
    }
    static constexpr int NR = 1, NI = 1;
    __device__ const double* raw_ptr(const FusedArgs& a, int) const { (void)a; return a.u[0]; }
    __device__ const double* in_ptr(const FusedArgs& a, int) const { return a.u0; }
    __device__ Raw raw_from(const double* v) const
    {
        Raw r;
        r.u = v[0];
        return r;
    }
    __device__ In in_from(const double* v) const
    {
        In in;
        in.u0 = v[0];
        return in;
    }
    __device__ void interior_k(const FusedArgs& a, long i, const Nb& nb, const Raw&, const In& in, double kx0,
                               double kx1, double ky0, double ky1, double kz0, double kz1, DDVec<2>& acc) const
    {
        const double s = smvp_k(nb, kx0, kx1, ky0, ky1, kz0, kz1);
        const double r = in.u0 - s;
        const float r32 = (float)r;
        a.r32[i] = r32;
        if (cheby) {
            const float p = r32 / theta32;
            a.p32[0][i] = p;
            a.d32[i] = p;
        } else {
            a.p32[0][i] = r32;
            a.d32[i] = 0.0f;
        }
        dd_add(acc.v[0], r * r);
        dd_add(acc.v[1], (double)r32 * (double)r32);
    }
    __device__ void control(const FusedArgs& a, const double* v)
    {
        if (a.timing) return;
        SolveState& s = *a.st;
        s.error = v[0];
        s.rro = v[1];
        s.pending_p = 0;
        s.pending_u = 0;
        s.par_p = 0;
        s.par_u = 0;
        s.n_inner = cheby ? 1 : 0;
        if (!isfinite(v[0])) s.nonfinite = 1;
    }
};

// FP32 CG sweep A: pending p = beta p + r and d += alpha p of the previous inner
// iteration, then w = A p and pw.
struct OpSweepA32 {
    static constexpr bool kReduce = true;
    using T = float;
    static constexpr int NV = 1;
    __device__ const float* coef_x(const FusedArgs& a) const { return a.kx32; }
    __device__ const float* coef_y(const FusedArgs& a) const { return a.ky32; }
    __device__ const float* coef_z(const FusedArgs& a) const { return a.kz32; }
    const float* pcur;
    float* pnew;
    float beta, alpha;
    int pend_p, pend_u;
    struct Raw {
        float p, r;
    };
    struct In {
        float d;
    };
    __device__ bool skip(const FusedArgs&) { return false; }
    __device__ void begin(const FusedArgs& a)
    {
        const SolveState& s = *a.st;
        pcur = a.p32[s.par_p];
        pnew = a.p32[s.par_p ^ 1];
        beta = (float)s.last_beta;
        alpha = (float)s.last_alpha;
        pend_p = s.pending_p;
        pend_u = s.pending_u;
    }
    __device__ Raw load_raw(const FusedArgs& a, long i) const
    {
        Raw r;
        r.p = pcur[i];
        r.r = pend_p ? a.r32[i] : 0.0f;
        return r;
    }
    __device__ float stage_raw(const Raw& r) const { return pend_p ? beta * r.p + r.r : r.p; }
    __device__ In load_in(const FusedArgs& a, long i) const
    {
        In in;
        in.d = pend_u ? a.d32[i] : 0.0f;
        return in;
    }
    static constexpr int NR = 2, NI = 1;
    __device__ const float* raw_ptr(const FusedArgs& a, int k) const
    {
        return k == 0 ? pcur : (pend_p ? a.r32 : nullptr);
    }
    __device__ const float* in_ptr(const FusedArgs& a, int) const { return pend_u ? a.d32 : nullptr; }
    __device__ Raw raw_from(const float* v) const
    {
        Raw r;
        r.p = v[0];
        r.r = pend_p ? v[1] : 0.0f;
        return r;
    }
    __device__ In in_from(const float* v) const
    {
        In in;
        in.d = pend_u ? v[0] : 0.0f;
        return in;
    }
    __device__ void interior_k(const FusedArgs& a, long i, const NbT<float>& nb, const Raw& rc, const In& in,
                               float kx0, float kx1, float ky0, float ky1, float kz0, float kz1,
                               DDVec<1>& acc) const
    {
        if (pend_u) a.d32[i] = in.d + alpha * rc.p;
        pnew[i] = nb.c;
        const float w = smvp_k(nb, kx0, kx1, ky0, ky1, kz0, kz1);
        a.w32[i] = w;
        dd_add(acc.v[0], (double)w * (double)nb.c);
    }
    // Ring kernels' vector-store form of interior_k: the same values, the lane's four cells
    // stored with one 16-byte store per array (d only when its update is pending).
    struct Out {
        float d, p, w;
    };
    __device__ Out interior_out(const NbT<float>& nb, const Raw& rc, const In& in, float kx0, float kx1, float ky0,
                                float ky1, float kz0, float kz1, DDVec<1>& acc, bool inner) const
    {
        Out o;
        o.d = in.d + alpha * rc.p;
        o.p = nb.c;
        o.w = smvp_k(nb, kx0, kx1, ky0, ky1, kz0, kz1);
        if (inner) dd_add(acc.v[0], (double)o.w * (double)nb.c);
        return o;
    }
    __device__ void store_vec(const FusedArgs& a, long i, const Out* o) const
    {
        static_assert(RingVec<OpSweepA32>::value == 4, "one float4 per array");
        const float d4[4] = {o[0].d, o[1].d, o[2].d, o[3].d}, p4[4] = {o[0].p, o[1].p, o[2].p, o[3].p},
                    w4[4] = {o[0].w, o[1].w, o[2].w, o[3].w};
        if (pend_u) st_vec(a.d32 + i, d4);
        st_vec(pnew + i, p4);
        st_vec(a.w32 + i, w4);
    }
    __device__ void store_one(const FusedArgs& a, long i, const Out& o) const
    {
        if (pend_u) a.d32[i] = o.d;
        pnew[i] = o.p;
        a.w32[i] = o.w;
    }
    __device__ void control(const FusedArgs& a, const double* v)
    {
        if (a.timing) return;
        SolveState& s = *a.st;
        s.pw = v[0];
        s.alpha = s.rro / v[0];
        s.par_p ^= 1;
        s.pending_p = 0;
        s.pending_u = 0;
        if (!isfinite(v[0])) s.nonfinite = 1;
    }
};

// FP32 Chebyshev iteration of the inner solve A d = r32 (the reference's ChebyIterate +
// ChebyCalcU with u0 -> r32, u -> d), the standard coefficient sequence from the first
// iteration on; the inner residual norm every 10 iterations decides the inner stop
// (sum r^2 < tol2) beside inner_max.
struct OpCheby32 {
    static constexpr bool kReduce = true;
    using T = float;
    static constexpr int NV = 1;
    __device__ const float* coef_x(const FusedArgs& a) const { return a.kx32; }
    __device__ const float* coef_y(const FusedArgs& a) const { return a.ky32; }
    __device__ const float* coef_z(const FusedArgs& a) const { return a.kz32; }
    const float* ucur;  // the iterate d
    float* unew;
    float* pcur;
    float* pnext;
    float al, be;
    int j, jmax, check;
    __device__ bool skip(const FusedArgs&) { return false; }
    __device__ void begin(const FusedArgs& a)
    {
        const SolveState& s = *a.st;
        ucur = a.dc32[s.par_u];
        unew = a.dc32[s.par_u ^ 1];
        pcur = a.p32[s.par_p];
        pnext = a.p32[s.par_p ^ 1];
        j = s.n_inner;
        jmax = s.inner_max;
        al = (float)a.ch_alphas[j - 1];
        be = (float)a.ch_betas[j - 1];
        check = (j % 10 == 0);
    }
    struct Raw {
        float d;
    };
    struct In {
        float rhs, p;
    };
    __device__ Raw load_raw(const FusedArgs&, long i) const
    {
        Raw r;
        r.d = ucur[i];
        return r;
    }
    __device__ float stage_raw(const Raw& r) const { return r.d; }
    __device__ In load_in(const FusedArgs& a, long i) const
    {
        In in;
        in.rhs = a.r32[i];
        in.p = pcur[i];
        return in;
    }
    static constexpr int NR = 1, NI = 2;
    __device__ const float* raw_ptr(const FusedArgs&, int) const { return ucur; }
    __device__ const float* in_ptr(const FusedArgs& a, int k) const { return k == 0 ? a.r32 : pcur; }
    __device__ Raw raw_from(const float* v) const
    {
        Raw r;
        r.d = v[0];
        return r;
    }
    __device__ In in_from(const float* v) const
    {
        In in;
        in.rhs = v[0];
        in.p = v[1];
        return in;
    }
    __device__ void interior_k(const FusedArgs&, long i, const NbT<float>& nb, const Raw&, const In& in, float kx0,
                               float kx1, float ky0, float ky1, float kz0, float kz1, DDVec<1>& acc) const
    {
        const float w = smvp_k(nb, kx0, kx1, ky0, ky1, kz0, kz1);
        const float r = in.rhs - w;
        const float p = al * in.p + be * r;
        pcur[i] = p;
        unew[i] = nb.c + p;
        if (check) dd_add(acc.v[0], (double)r * (double)r);
    }
    // Ring kernels' vector-store form of interior_k: the lane's four cells of p and of the
    // new iterate stored with one 16-byte store each.
    struct Out {
        float p, u;
    };
    __device__ Out interior_out(const NbT<float>& nb, const Raw&, const In& in, float kx0, float kx1, float ky0,
                                float ky1, float kz0, float kz1, DDVec<1>& acc, bool inner) const
    {
        const float w = smvp_k(nb, kx0, kx1, ky0, ky1, kz0, kz1);
        const float r = in.rhs - w;
        Out o;
        o.p = al * in.p + be * r;
        o.u = nb.c + o.p;
        if (check && inner) dd_add(acc.v[0], (double)r * (double)r);
        return o;
    }
    __device__ void store_vec(const FusedArgs&, long i, const Out* o) const
    {
        const float p4[4] = {o[0].p, o[1].p, o[2].p, o[3].p}, u4[4] = {o[0].u, o[1].u, o[2].u, o[3].u};
        st_vec(pcur + i, p4);
        st_vec(unew + i, u4);
    }
    __device__ void store_one(const FusedArgs&, long i, const Out& o) const
    {
        pcur[i] = o.p;
        unew[i] = o.u;
    }
    __device__ static void finish(const FusedArgs& a, SolveState& s, bool checked, double rr)
    {
        if (checked) s.rrn = rr;
        // Healthy Chebyshev: sum r^2 <= 4 rho^(2k) sum r0^2.  Far above that (1e4) after 50
        // iterations, or growing, means the spectrum estimate missed low modes.
        const bool diverged = checked && (!(rr <= 100.0 * s.rro) ||
                                          (s.n_inner >= 50 && rr > 1e4 * s.rro * pow(s.cheby_rho2, (double)s.n_inner)));
        if (diverged) s.inner_diverged = 1;
        const bool stop = (checked && (rr < s.tol2 || diverged)) || s.n_inner >= s.inner_max;
        s.cont = !stop;
        if (a.use_handle) cudaGraphSetConditional(a.handle, stop ? 0u : 1u);
    }
    __device__ void control(const FusedArgs& a, const double* v)
    {
        if (a.timing) return;
        SolveState& s = *a.st;
        s.par_u ^= 1;
        s.n_inner = j + 1;
        finish(a, s, check != 0, v[0]);
    }
    // Passes of nit iterations: none of iterations j .. j + nit - 2 is a check and the pass
    // stays below the correction's limit.
    __device__ bool pass_ok(const FusedArgs&, int nit) const
    {
        for (int k = 0; k < nit - 1; ++k)
            if ((j + k) % 10 == 0) return false;
        return j + nit - 1 < jmax;
    }
    __device__ void pass_coefs(const FusedArgs& a, int l, float& al_l, float& be_l) const
    {
        al_l = (float)a.ch_alphas[j - 1 + l];
        be_l = (float)a.ch_betas[j - 1 + l];
    }
    __device__ bool pass_check(const FusedArgs&, int nit) const { return (j + nit - 1) % 10 == 0; }
    __device__ const float* pair_rhs(const FusedArgs& a) const { return a.r32; }
    __device__ const float* pair_mi(const FusedArgs&) const { return nullptr; }
    __device__ void pass_control(const FusedArgs& a, const double* v, int nit, bool check_last) const
    {
        if (a.timing) return;
        SolveState& s = *a.st;
        s.par_u ^= 1;
        s.par_p ^= 1;
        s.n_inner = j + nit;
        finish(a, s, check_last, v[0]);
    }
};

// FP32 CG sweep B: r -= alpha w, rr; beta, and the inner loop test: stop when the inner
// residual has dropped below tol2 (inner_tol^2 times its start) or after inner_max.
__global__ void __launch_bounds__(256) k_cg32_sweep_b(FusedArgs a)
{
    const SolveState& s = *a.st;
    const float alpha = (float)s.alpha;
    float* __restrict__ R = a.r32;
    const float* __restrict__ W = a.w32;
    DDVec<1> acc;
    acc.zero();
    walk_quads(a.g, [&](long i, int n) {
        if (n == 4) {
            const float4 r4 = *reinterpret_cast<const float4*>(R + i);
            const float4 w4 = *reinterpret_cast<const float4*>(W + i);
            const float r0 = r4.x - alpha * w4.x, r1 = r4.y - alpha * w4.y;
            const float r2 = r4.z - alpha * w4.z, r3 = r4.w - alpha * w4.w;
            *reinterpret_cast<float4*>(R + i) = make_float4(r0, r1, r2, r3);
            dd_add(acc.v[0], (double)r0 * (double)r0);
            dd_add(acc.v[0], (double)r1 * (double)r1);
            dd_add(acc.v[0], (double)r2 * (double)r2);
            dd_add(acc.v[0], (double)r3 * (double)r3);
        } else {
            for (int k = 0; k < n; ++k) {
                const float r0 = R[i + k] - alpha * W[i + k];
                R[i + k] = r0;
                dd_add(acc.v[0], (double)r0 * (double)r0);
            }
        }
    });
    grid_reduce_then<1>(acc, a.red, [&](const double* v) {
        if (a.timing) return;
        SolveState& st = *a.st;
        st.rrn = v[0];
        st.beta = st.rrn / st.rro;
        st.rro = st.rrn;
        st.last_alpha = st.alpha;
        st.last_beta = st.beta;
        st.pending_p = 1;
        st.pending_u = 1;
        st.n_inner = st.n_inner + 1;
        // The inner CG's scalars feed the Lanczos eigenvalue estimate of the Chebyshev
        // corrections (indexed 1.., as the FP64 loop stores them).
        a.cg_alphas[st.n_inner] = st.alpha;
        a.cg_betas[st.n_inner] = st.beta;
        if (!isfinite(v[0])) st.nonfinite = 1;
        const bool at_switch = st.switch_err > 0.0 && st.n_inner >= st.switch_min && v[0] <= st.switch_err;
        const int cont = isfinite(v[0]) && v[0] >= st.tol2 && st.n_inner < st.inner_max && !at_switch;
        st.cont = cont;
        if (a.use_handle) cudaGraphSetConditional(a.handle, cont ? 1u : 0u);
    });
}

// u += d in FP64, after the pending d += alpha p of the last inner iteration.
// The FP32 inner PPCG's CGCalcUr + PPCGInitSd (the FP32 form of k_ppcg_sweep_b, no
// preconditioner): d += alpha p, r -= alpha w (into w when the two-step passes start there),
// sd = r / theta into sd32[0].
__global__ void __launch_bounds__(256) k_ppcg32_sweep_b(FusedArgs a)
{
    const SolveState& s = *a.st;
    const float alpha = (float)s.alpha, theta = (float)s.theta;
    const float* __restrict__ P = a.p32[s.par_p];
    float* __restrict__ D = a.d32;
    const float* R = a.r32;
    const float* W = a.w32;
    float* RD = a.r_in_w ? a.w32 : a.r32;
    float* __restrict__ SD = a.sd32[0];
    walk_quads(a.g, [&](long i, int n) {
        if (n == 4) {
            const float4 d4 = *reinterpret_cast<const float4*>(D + i), p4 = *reinterpret_cast<const float4*>(P + i);
            const float4 r4 = *reinterpret_cast<const float4*>(R + i), w4 = *reinterpret_cast<const float4*>(W + i);
            *reinterpret_cast<float4*>(D + i) =
                make_float4(d4.x + alpha * p4.x, d4.y + alpha * p4.y, d4.z + alpha * p4.z, d4.w + alpha * p4.w);
            const float r0 = r4.x - alpha * w4.x, r1 = r4.y - alpha * w4.y;
            const float r2 = r4.z - alpha * w4.z, r3 = r4.w - alpha * w4.w;
            *reinterpret_cast<float4*>(RD + i) = make_float4(r0, r1, r2, r3);
            *reinterpret_cast<float4*>(SD + i) = make_float4(r0 / theta, r1 / theta, r2 / theta, r3 / theta);
        } else {
            for (int k = 0; k < n; ++k) {
                D[i + k] = D[i + k] + alpha * P[i + k];
                const float r = R[i + k] - alpha * W[i + k];
                RD[i + k] = r;
                SD[i + k] = r / theta;
            }
        }
    });
}

__global__ void __launch_bounds__(256) k_dc_update(FusedArgs a)
{
    const SolveState& s = *a.st;
    const float alpha = (float)s.last_alpha;
    const int pend = s.inner_cheby ? 0 : s.pending_u;
    const float* __restrict__ P = a.p32[s.par_p];
    const float* __restrict__ D = s.inner_cheby == 1 ? a.dc32[s.par_u] : a.d32;
    walk_pairs(a.g, [&](long i, bool two) {
        const int n = two ? 2 : 1;
        for (int k = 0; k < n; ++k) {
            float d = D[i + k];
            if (pend) d = d + alpha * P[i + k];
            a.u[0][i + k] = a.u[0][i + k] + (double)d;
        }
    });
}

// ------------------------------------------------------------------ flush

// Applies what the fused CG/PPCG loop left pending so that u and p hold exactly what the
// reference's per-iteration calls would have left: u += last_alpha p, p = last_beta p +
// (z|r), both in place on the current buffers.
__global__ void __launch_bounds__(BLOCK) k_flush(FusedArgs a, Box inner)
{
    const SolveState& s = *a.st;
    if (!s.pending_p && !s.pending_u) return;
    double* p = a.p[s.par_p];
    const double alpha = s.last_alpha, beta = s.last_beta;
    const int pu = s.pending_u, pp = s.pending_p, precond = s.precond;
    const Geom& g = a.g;
    walk(inner, [&](int kk, int jj, int ii) {
        const long i = fidx(g, kk, jj, ii);
        const double po = p[i];
        if (pu) a.u[0][i] = a.u[0][i] + alpha * po;
        if (pp) p[i] = beta * po + (precond ? a.z[i] : a.r[i]);
    });
}

__global__ void k_clear_pending(SolveState* s)
{
    s->pending_p = 0;
    s->pending_u = 0;
}

}  // namespace tea
