// Fused kernels of the whole-solve path (ext_tea_leaf_solve_).
//
// One chunk, every face external.  The reference keeps each halo equal to the
// reflection of the interior whenever a stencil reads it (update_halo after every
// iteration, tealeaf_2d/tea_solve.f90:489, 632, 704), so these kernels read a
// neighbour outside the inner domain from its reflected interior cell instead of
// from the halo: same value, same arithmetic, no halo maintenance inside the loop.
//
// Stencil kernels stage the stencil operand for a tile plus a one-cell ring in shared
// memory (computing it on the way in where it is itself an update, e.g. CG's
// p = beta p + r), then apply the operator from shared memory.  2D tiles are 32 x 32
// cells for 256 threads; 3D tiles are 32 x 8 cells marching through a z segment with
// four rotating planes.  Buffers that a sweep both reads at neighbours and rewrites
// (p, u, sd) are double-buffered.
//
// Scalar recurrences (alpha = rro/pw, beta = rrn/rro, ...) and the loop test of
// tea_leaf() run in the last block of the reducing kernel, so one iteration is two
// (CG), one (Chebyshev, Jacobi) or 2 + inner-steps (PPCG) launches, captured in a
// CUDA graph whose while-node reads the continue flag set there.
#pragma once

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
    int timing;  // measurement launches: the last block leaves the solve state untouched
};

constexpr int FT_X = 32;
constexpr int FT_Y2 = 32;   // 2D tile height
constexpr int FT_Y3 = 8;    // 3D tile height
constexpr int FBLOCK = 256;

// Reflection of a padded index into the inner domain (depth 1 and 2): HALO_PAD-1-f
// maps to HALO_PAD+f and N-HALO_PAD+f to N-HALO_PAD-1-f, as UpdateHalo copies them.
__device__ __forceinline__ int refl(int k, int n)
{
    return k < HALO_PAD ? 2 * HALO_PAD - 1 - k : (k >= n - HALO_PAD ? 2 * (n - HALO_PAD) - 1 - k : k);
}

struct Nb {
    double c, xm, xp, ym, yp, zm, zp;
};

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

// Op interface:
//   static constexpr bool kReduce;
//   __device__ void begin(const FusedArgs&)                      -- read scalars
//   __device__ double stage(const FusedArgs&, long i)             -- operand at a (reflected) cell
//   __device__ void interior(const FusedArgs&, long i, const Nb&, DD& acc)
//   __device__ void control(const FusedArgs&, double v)           -- last block, lane 0
//   __device__ bool skip(const FusedArgs&)                        -- whole launch is a no-op

template <class Op>
__global__ void __launch_bounds__(FBLOCK) k_stencil2d(FusedArgs a)
{
    constexpr int SX = FT_X + 2, SY = FT_Y2 + 2;
    __shared__ double s_op[SY][SX];
    Op op;
    if (op.skip(a)) return;
    op.begin(a);
    const Geom& g = a.g;
    DDVec<1> acc;
    acc.zero();
    const int tid = threadIdx.x + threadIdx.y * FT_X;
    for (long t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
        const int tx = (int)(t % a.tiles_x), ty = (int)(t / a.tiles_x);
        const int x0 = HALO_PAD + tx * FT_X, y0 = HALO_PAD + ty * FT_Y2;
        for (int s = tid; s < SX * SY; s += FBLOCK) {
            const int lx = s % SX, ly = s / SX;
            const int kk = x0 - 1 + lx, jj = y0 - 1 + ly;
            if (kk <= g.X - 2 && jj <= g.Y - 2) s_op[ly][lx] = op.stage(a, fidx(g, refl(kk, g.X), refl(jj, g.Y), 0));
        }
        __syncthreads();
#pragma unroll
        for (int c = 0; c < FT_Y2 / 8; ++c) {
            const int lx = (int)threadIdx.x + 1, ly = (int)threadIdx.y + 8 * c + 1;
            const int kk = x0 + (int)threadIdx.x, jj = y0 + (int)threadIdx.y + 8 * c;
            if (kk < g.X - HALO_PAD && jj < g.Y - HALO_PAD) {
                Nb nb;
                nb.c = s_op[ly][lx];
                nb.xm = s_op[ly][lx - 1];
                nb.xp = s_op[ly][lx + 1];
                nb.ym = s_op[ly - 1][lx];
                nb.yp = s_op[ly + 1][lx];
                nb.zm = nb.zp = 0.0;
                op.interior(a, fidx(g, kk, jj, 0), nb, acc.v[0]);
            }
        }
        __syncthreads();
    }
    if (Op::kReduce) grid_reduce_then<1>(acc, a.red, [&](const double* v) { op.control(a, v[0]); });
}

template <class Op>
__global__ void __launch_bounds__(FBLOCK) k_stencil3d(FusedArgs a)
{
    constexpr int SX = FT_X + 2, SY = FT_Y3 + 2;
    __shared__ double s_op[4][SY][SX];
    Op op;
    if (op.skip(a)) return;
    op.begin(a);
    const Geom& g = a.g;
    DDVec<1> acc;
    acc.zero();
    const int tid = threadIdx.x + threadIdx.y * FT_X;
    const long txy = (long)a.tiles_x * a.tiles_y;
    for (long t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
        const int zs = (int)(t / txy);
        const long rxy = t % txy;
        const int tx = (int)(rxy % a.tiles_x), ty = (int)(rxy / a.tiles_x);
        const int x0 = HALO_PAD + tx * FT_X, y0 = HALO_PAD + ty * FT_Y3;
        const int z0 = HALO_PAD + zs * a.zseg;
        const int z1 = min(z0 + a.zseg, g.Z - HALO_PAD);
        auto stage_plane = [&](int ii) {
            double(*pl)[SX] = s_op[ii & 3];
            const int ri = refl(ii, g.Z);
            for (int s = tid; s < SX * SY; s += FBLOCK) {
                const int lx = s % SX, ly = s / SX;
                const int kk = x0 - 1 + lx, jj = y0 - 1 + ly;
                if (kk <= g.X - 2 && jj <= g.Y - 2) pl[ly][lx] = op.stage(a, fidx(g, refl(kk, g.X), refl(jj, g.Y), ri));
            }
        };
        stage_plane(z0 - 1);
        stage_plane(z0);
        for (int ii = z0; ii < z1; ++ii) {
            stage_plane(ii + 1);
            __syncthreads();
            const int lx = (int)threadIdx.x + 1, ly = (int)threadIdx.y + 1;
            const int kk = x0 + (int)threadIdx.x, jj = y0 + (int)threadIdx.y;
            if (kk < g.X - HALO_PAD && jj < g.Y - HALO_PAD) {
                const double(*pm)[SX] = s_op[(ii - 1) & 3];
                const double(*pc)[SX] = s_op[ii & 3];
                const double(*pp)[SX] = s_op[(ii + 1) & 3];
                Nb nb;
                nb.c = pc[ly][lx];
                nb.xm = pc[ly][lx - 1];
                nb.xp = pc[ly][lx + 1];
                nb.ym = pc[ly - 1][lx];
                nb.yp = pc[ly + 1][lx];
                nb.zm = pm[ly][lx];
                nb.zp = pp[ly][lx];
                op.interior(a, fidx(g, kk, jj, ii), nb, acc.v[0]);
            }
        }
        __syncthreads();
    }
    if (Op::kReduce) grid_reduce_then<1>(acc, a.red, [&](const double* v) { op.control(a, v[0]); });
}

// 2D register streaming: a block of SW warps covers 32*SW adjacent columns and marches
// down SY rows; each lane owns one column and keeps the staged operand of rows j-1, j,
// j+1 in registers.  x-neighbours come from the adjacent lanes by shuffle; the two lanes
// at the warp's edges stage their outside neighbour themselves.  No shared memory and no
// block barrier: every array is read once per cell (plus the edge columns and one row
// above and below each column segment, which hit L2).
constexpr int SW = 4;      // warps per block
constexpr int SY = 32;     // rows per column segment
constexpr int SBLOCK = 32 * SW;

template <class Op>
__global__ void __launch_bounds__(SBLOCK) k_stream2d(FusedArgs a)
{
    Op op;
    if (op.skip(a)) return;
    op.begin(a);
    const Geom& g = a.g;
    DDVec<1> acc;
    acc.zero();
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int xlast = g.X - HALO_PAD - 1;  // last inner column
    const int ylast = g.Y - HALO_PAD - 1;
    for (long t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
        const int tx = (int)(t % a.tiles_x), ty = (int)(t / a.tiles_x);
        const int kk = HALO_PAD + tx * SBLOCK + warp * 32 + lane;
        if (HALO_PAD + tx * SBLOCK + warp * 32 > xlast) continue;  // whole warp outside: uniform
        const bool active = kk <= xlast;
        const int kc = min(kk, xlast);                 // inactive lanes shadow the last column
        const bool edge = lane == 0 || lane == 31;
        const int ke = lane == 0 ? refl(kc - 1, g.X) : refl(min(kc + 1, xlast + 1), g.X);
        const int j0 = HALO_PAD + ty * SY;
        const int j1 = min(j0 + SY, ylast + 1);
        double cm = op.stage(a, fidx(g, kc, refl(j0 - 1, g.Y), 0));
        double cc = op.stage(a, fidx(g, kc, j0, 0));
        for (int jj = j0; jj < j1; ++jj) {
            const double cp = op.stage(a, fidx(g, kc, refl(jj + 1, g.Y), 0));
            double e = 0.0;
            if (edge) e = op.stage(a, fidx(g, ke, jj, 0));
            const double up = __shfl_up_sync(0xffffffffu, cc, 1);
            const double dn = __shfl_down_sync(0xffffffffu, cc, 1);
            if (active) {
                Nb nb;
                nb.c = cc;
                nb.xm = lane == 0 ? e : up;
                nb.xp = lane == 31 ? e : dn;
                nb.ym = cm;
                nb.yp = cp;
                nb.zm = nb.zp = 0.0;
                op.interior(a, fidx(g, kk, jj, 0), nb, acc.v[0]);
            }
            cm = cc;
            cc = cp;
        }
    }
    if (Op::kReduce) grid_reduce_then<1>(acc, a.red, [&](const double* v) { op.control(a, v[0]); });
}

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
    struct Bundle {
        In in;
        double kx, ky, kxe;
    };
    Op op;
    if (op.skip(a)) return;
    op.begin(a);
    const Geom& g = a.g;
    const double* __restrict__ KX = a.kx;
    const double* __restrict__ KY = a.ky;
    DDVec<1> acc;
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
            const long i = fidx(g, kq, jj, 0);
            b.in = op.load_in(a, fidx(g, kc, jj, 0));
            b.kx = KX[i];
            b.ky = KY[fidx(g, kc, jj, 0)];
            b.kxe = lane == 31 ? KX[fidx(g, min(kk + 1, xlast + 1), jj, 0)] : 0.0;
            return b;
        };
        Raw rc = op.load_raw(a, fidx(g, kc, j0, 0));
        Raw rp = op.load_raw(a, fidx(g, kc, refl(j0 + 1, g.Y), 0));
        double sm = op.stage_raw(op.load_raw(a, fidx(g, kc, refl(j0 - 1, g.Y), 0)));
        double sc = op.stage_raw(rc);
        Bundle bc = bundle(j0);
        Bundle bn = bundle(j0 + 1);
        Raw rec;
        if (edge) rec = op.load_raw(a, fidx(g, ke, j0, 0));
        for (int jj = j0; jj < j1; ++jj) {
            // Prefetch row jj+2 (operand, interior bundle) and the edge operand of row jj+1.
            const Raw rpp = op.load_raw(a, fidx(g, kc, refl(min(jj + 2, ylast + 2), g.Y), 0));
            const Bundle bnn = bundle(min(jj + 2, ylast + 1));
            Raw ren;
            if (edge) ren = op.load_raw(a, fidx(g, ke, min(jj + 1, ylast), 0));
            const double sp = op.stage_raw(rp);
            const double e = edge ? op.stage_raw(rec) : 0.0;
            const double up = __shfl_up_sync(0xffffffffu, sc, 1);
            const double dn = __shfl_down_sync(0xffffffffu, sc, 1);
            const double kxr = __shfl_down_sync(0xffffffffu, bc.kx, 1);
            if (active) {
                Nb nb;
                nb.c = sc;
                nb.xm = lane == 0 ? e : up;
                nb.xp = lane == 31 ? e : dn;
                nb.ym = sm;
                nb.yp = sp;
                nb.zm = nb.zp = 0.0;
                const double kx1 = lane == 31 ? bc.kxe : kxr;
                op.interior2(a, fidx(g, kk, jj, 0), nb, rc, bc.in, bc.kx, kx1, bc.ky, bn.ky, acc.v[0]);
            }
            sm = sc;
            sc = sp;
            rc = rp;
            rp = rpp;
            bc = bn;
            bn = bnn;
            if (edge) rec = ren;
        }
    }
    if (Op::kReduce) grid_reduce_then<1>(acc, a.red, [&](const double* v) { op.control(a, v[0]); });
}

#if TEA_DIM == 2
#define TEA_STENCIL k_pipe2d
#define TEA_STENCIL_BLOCK dim3(SBLOCK)
#else
#define TEA_STENCIL k_stencil3d
#define TEA_STENCIL_BLOCK dim3(FT_X, FBLOCK / FT_X)
#endif

// ------------------------------------------------------------------ CG / PPCG sweep A

// Applies the pending p update of the previous iteration (CGCalcP,
// tealeaf_2d/ext_cg_kernel.hpp:301-310, and for CG the deferred u += alpha p of CGCalcUr
// :251), then w = A p and pw = sum w.p (CGCalcW :177-189).  The new p goes to the other
// p buffer.
struct OpSweepA {
    static constexpr bool kReduce = true;
    const double* pcur;
    double* pnew;
    double beta, alpha;
    int pend_p, pend_u, precond;
    __device__ bool skip(const FusedArgs&) { return false; }
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
    __device__ double stage(const FusedArgs& a, long i)
    {
        const double p = pcur[i];
        if (!pend_p) return p;
        return beta * p + (precond ? a.z[i] : a.r[i]);
    }
    __device__ void interior(const FusedArgs& a, long i, const Nb& nb, DD& acc)
    {
        if (pend_u) a.u[0][i] = a.u[0][i] + alpha * pcur[i];
        pnew[i] = nb.c;
        const double w = smvp_nb(nb, a.kx, a.ky, a.kz, i, a.g.pitch, a.g.page);
        a.w[i] = w;
        dd_add(acc, w * nb.c);
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
    __device__ void interior2(const FusedArgs& a, long i, const Nb& nb, const Raw& rc, const In& in, double kx0,
                              double kx1, double ky0, double ky1, DD& acc) const
    {
        if (pend_u) a.u[0][i] = in.u + alpha * rc.p;
        pnew[i] = nb.c;
        const double w = (1.0 + (kx1 + kx0) + (ky1 + ky0)) * nb.c - (kx1 * nb.xp + kx0 * nb.xm)
            - (ky1 * nb.yp + ky0 * nb.ym);
        a.w[i] = w;
        dd_add(acc, w * nb.c);
    }
    __device__ void control(const FusedArgs& a, double pw)
    {
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

__device__ __forceinline__ double2 ld2(const double* p) { return *reinterpret_cast<const double2*>(p); }
__device__ __forceinline__ void st2(double* p, double a, double b) { *reinterpret_cast<double2*>(p) = make_double2(a, b); }

// CGCalcUr without the u update (deferred to the next sweep A): r -= alpha w, z = Mi r,
// rrn = sum r.r or r.z; then beta = rrn/rro and the end-of-iteration test.
__global__ void __launch_bounds__(256) k_cg_sweep_b(FusedArgs a)
{
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
__global__ void __launch_bounds__(BLOCK) k_ppcg_sweep_b(FusedArgs a, Box inner)
{
    const SolveState& s = *a.st;
    const double alpha = s.alpha, theta = s.theta;
    const int precond = s.precond;
    const double* __restrict__ p = a.p[s.par_p];
    const Geom& g = a.g;
    walk(inner, [&](int kk, int jj, int ii) {
        const long i = fidx(g, kk, jj, ii);
        a.u[0][i] = a.u[0][i] + alpha * p[i];
        const double r = a.r[i] - alpha * a.w[i];
        a.r[i] = r;
        double m = r;
        if (precond) {
            m = a.mi[i] * r;
            a.z[i] = m;
        }
        a.sd[0][i] = m / theta;
    });
}

// One PPCG inner step k (1-based): PPCGCalcU (r -= A sd, u += sd,
// tealeaf_2d/ext_ppcg_kernel.hpp:37-65) then PPCGCalcSd (:68-100) into the other sd
// buffer.  The last step also forms sum r.r (ext_calculate_2norm_, tea_solve.f90:346)
// and runs the end of the outer iteration (beta, calc_p deferred, EXIT test).
template <bool LAST>
struct OpPPCGInner {
    static constexpr bool kReduce = LAST;
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
    __device__ double stage(const FusedArgs&, long i) { return sdc[i]; }
    __device__ void interior(const FusedArgs& a, long i, const Nb& nb, DD& acc)
    {
        const double s = smvp_nb(nb, a.kx, a.ky, a.kz, i, a.g.pitch, a.g.page);
        const double r = a.r[i] - s;
        a.r[i] = r;
        a.u[0][i] = a.u[0][i] + nb.c;
        sdn[i] = al * nb.c + be * (precond ? a.mi[i] * r : r);
        if (LAST) dd_add(acc, r * r);
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
    __device__ void interior2(const FusedArgs& a, long i, const Nb& nb, const Raw&, const In& in, double kx0,
                              double kx1, double ky0, double ky1, DD& acc) const
    {
        const double s = (1.0 + (kx1 + kx0) + (ky1 + ky0)) * nb.c - (kx1 * nb.xp + kx0 * nb.xm)
            - (ky1 * nb.yp + ky0 * nb.ym);
        const double r = in.r - s;
        a.r[i] = r;
        a.u[0][i] = in.u + nb.c;
        sdn[i] = al * nb.c + be * (precond ? in.mi * r : r);
        if (LAST) dd_add(acc, r * r);
    }
    __device__ void control(const FusedArgs& a, double rrn)
    {
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

// ------------------------------------------------------------------ Chebyshev

// ChebyIterate + ChebyCalcU (tealeaf_2d/ext_cheby_kernel.hpp:50-115) in one sweep: the
// operator reads u_old, u_new = u_old + p goes to the other u buffer.  sum r.r is formed
// on the iterations where tea_leaf() checks it (n >= est_itc and MOD(n,10) == 0,
// tealeaf_2d/tea_solve.f90:260).
struct OpCheby {
    static constexpr bool kReduce = true;
    const double* ucur;
    double* unew;
    double al, be;
    int precond, check;
    __device__ bool skip(const FusedArgs&) { return false; }
    __device__ void begin(const FusedArgs& a)
    {
        const SolveState& s = *a.st;
        ucur = a.u[s.par_u];
        unew = a.u[s.par_u ^ 1];
        const int step = s.cheby_calc_steps - 1;
        al = a.ch_alphas[step];
        be = a.ch_betas[step];
        precond = s.precond;
        check = (s.n >= s.est_itc) && (s.n % 10 == 0);
    }
    __device__ double stage(const FusedArgs&, long i) { return ucur[i]; }
    __device__ void interior(const FusedArgs& a, long i, const Nb& nb, DD& acc)
    {
        const double w = smvp_nb(nb, a.kx, a.ky, a.kz, i, a.g.pitch, a.g.page);
        const double r = a.u0[i] - w;
        const double p = al * a.p[0][i] + be * (precond ? a.mi[i] * r : r);
        a.p[0][i] = p;
        unew[i] = nb.c + p;
        if (check) dd_add(acc, r * r);
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
        in.p = a.p[0][i];
        in.mi = precond ? a.mi[i] : 0.0;
        return in;
    }
    __device__ void interior2(const FusedArgs& a, long i, const Nb& nb, const Raw&, const In& in, double kx0,
                              double kx1, double ky0, double ky1, DD& acc) const
    {
        const double w = (1.0 + (kx1 + kx0) + (ky1 + ky0)) * nb.c - (kx1 * nb.xp + kx0 * nb.xm)
            - (ky1 * nb.yp + ky0 * nb.ym);
        const double r = in.u0 - w;
        const double p = al * in.p + be * (precond ? in.mi * r : r);
        a.p[0][i] = p;
        unew[i] = nb.c + p;
        if (check) dd_add(acc, r * r);
    }
    __device__ void control(const FusedArgs& a, double rr)
    {
        if (a.timing) return;
        SolveState& s = *a.st;
        s.par_u ^= 1;
        if (check) s.error = rr;
        s.cheby_calc_steps = s.cheby_calc_steps + 1;
        end_iteration(a, s, PHASE_CHEBY);
    }
};

// ------------------------------------------------------------------ Jacobi

// JacobiCopyU + JacobiSolve (tealeaf_2d/ext_jacobi_kernel.hpp:66-117) with u
// double-buffered instead of copied: u_new from the staged u_old, error = sum|u_new-u_old|.
struct OpJacobi {
    static constexpr bool kReduce = true;
    const double* ucur;
    double* unew;
    __device__ bool skip(const FusedArgs&) { return false; }
    __device__ void begin(const FusedArgs& a)
    {
        const SolveState& s = *a.st;
        ucur = a.u[s.par_u];
        unew = a.u[s.par_u ^ 1];
    }
    __device__ double stage(const FusedArgs&, long i) { return ucur[i]; }
    __device__ void interior(const FusedArgs& a, long i, const Nb& nb, DD& acc)
    {
        const double* __restrict__ kx = a.kx;
        const double* __restrict__ ky = a.ky;
        const long px = a.g.pitch;
#if TEA_DIM == 2
        const double un = (a.u0[i] + (kx[i + 1] * nb.xp + kx[i] * nb.xm) + (ky[i + px] * nb.yp + ky[i] * nb.ym))
            / (1.0 + (kx[i] + kx[i + 1]) + (ky[i] + ky[i + px]));
#else
        const double* __restrict__ kz = a.kz;
        const long pg = a.g.page;
        const double un = (a.u0[i] + (kx[i + 1] * nb.xp + kx[i] * nb.xm) + (ky[i + px] * nb.yp + ky[i] * nb.ym)
                           + (kz[i + pg] * nb.zp + kz[i] * nb.zm))
            / (1.0 + (kx[i] + kx[i + 1]) + (ky[i] + ky[i + px]) + (kz[i] + kz[i + pg]));
#endif
        unew[i] = un;
        dd_add(acc, fabs(un - nb.c));
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
    __device__ void interior2(const FusedArgs&, long i, const Nb& nb, const Raw&, const In& in, double kx0,
                              double kx1, double ky0, double ky1, DD& acc) const
    {
        const double un = (in.u0 + (kx1 * nb.xp + kx0 * nb.xm) + (ky1 * nb.yp + ky0 * nb.ym))
            / (1.0 + (kx0 + kx1) + (ky0 + ky1));
        unew[i] = un;
        dd_add(acc, fabs(un - nb.c));
    }
    __device__ void control(const FusedArgs& a, double err)
    {
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
    const double* ucur;
    __device__ bool skip(const FusedArgs& a) { return a.st->resid_pending == 0; }
    __device__ void begin(const FusedArgs& a) { ucur = a.u[a.st->par_u]; }
    __device__ double stage(const FusedArgs&, long i) { return ucur[i]; }
    __device__ void interior(const FusedArgs& a, long i, const Nb& nb, DD& acc)
    {
        const double s = smvp_nb(nb, a.kx, a.ky, a.kz, i, a.g.pitch, a.g.page);
        const double r = a.u0[i] - s;
        a.r[i] = r;
        dd_add(acc, r * r);
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
    __device__ void interior2(const FusedArgs& a, long i, const Nb& nb, const Raw&, const In& in, double kx0,
                              double kx1, double ky0, double ky1, DD& acc) const
    {
        const double s = (1.0 + (kx1 + kx0) + (ky1 + ky0)) * nb.c - (kx1 * nb.xp + kx0 * nb.xm)
            - (ky1 * nb.yp + ky0 * nb.ym);
        const double r = in.u0 - s;
        a.r[i] = r;
        dd_add(acc, r * r);
    }
    __device__ void control(const FusedArgs& a, double rr)
    {
        if (a.timing) return;
        SolveState& s = *a.st;
        s.error = rr;
        s.resid_pending = 0;
        end_iteration(a, s, PHASE_JACOBI);
    }
};

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
