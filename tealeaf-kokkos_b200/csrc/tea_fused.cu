// ext_tea_leaf_solve_: the whole implicit solve of one timestep on the device.
//
// Follows tea_leaf() (tealeaf_2d/tea_solve.f90:36-605; 3D :36-653) step for step.  The
// once-per-solve parts -- set-up, the Chebyshev/PPCG switch with its eigenvalue estimate
// (host FP64, tea_eigen.h), the first Chebyshev step and the first PPCG outer iteration,
// the exact-residual check and the finalise -- call the same per-call kernels as the ext_*
// entry points.  The iteration loops run as CUDA graphs whose body is one iteration of
// fused kernels (tea_fused.cuh) inside a while-node; the scalars and the EXIT test live on
// the device.  Results (fields, iteration counts, errors) equal the per-call sequence that
// the driver would make bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/tea_b200.h"
#if TEA_DIM == 2
#include "../../include/tea_ext_2d.h"
#else
#include "../../include/tea_ext_3d.h"
#endif
#include "../driver/tea_eigen.h"
#include "tea_fused.cuh"

#define TEA_EXPORT extern "C" __attribute__((visibility("default")))

namespace tea {

Chunk* get_chunk(const int* chunk);
int ws_predict_into(Chunk* c, double* u_out);  // tea_warmstart.cu
void sync(Chunk* c);
void update_halo(Chunk* c, const int* neighbours, const int* fields, int depth);

namespace {

enum {
    LOOP_CG = 0, LOOP_CHEBY = 1, LOOP_PPCG = 2, LOOP_JACOBI = 3, LOOP_CG32 = 4, LOOP_CHEBY32 = 5, LOOP_PPCG32 = 6,
    LOOP_COUNT = 7
};

struct Loop {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int key = -1;
};

struct RingLaunch {
    int blocks = 0, rows = 0;
};
constexpr int RING_OPS = 9;

struct Fused {
    SolveState* d_st = nullptr;
    SolveState* h_st = nullptr;  // pinned
    double* alt[3] = {nullptr, nullptr, nullptr};  // allocations of u, p, sd second buffers
    float* alloc32[10] = {};  // FP32 arrays of the defect-correction form (allocated on first use)
    double *d_cg_alphas = nullptr, *d_cg_betas = nullptr;
    double *d_ch_alphas = nullptr, *d_ch_betas = nullptr;
    int cap = 0;  // entries of the coefficient arrays
    FusedArgs base{};
    int stencil_blocks = 0, point_blocks = 0, pair_blocks = 0, quad_blocks = 0;
    RingLaunch ring[RING_OPS];  // grid and segment rows of k_ring2d per sweep (2D)
    RingLaunch pair;            // k_cheby2_ring2d<OpCheby> (2D); blocks 0: one iteration per launch
    RingLaunch pair32;          // k_cheby2_ring2d<OpCheby32> (2D)
    RingLaunch quad;            // k_cheby4_ring2d<OpCheby> (2D); blocks 0: pairs only
    RingLaunch quadp;           // the same with the preconditioner (mi staged: more shared memory)
    RingLaunch quad32;          // k_cheby4_ring2d<OpCheby32> (2D)
    RingLaunch ring3[RING_OPS]; // grid and z-segment planes of k_ring3d per sweep (3D)
    RingLaunch ppcg2;           // k_ppcg2_ring3d (3D) / k_ppcg2_ring2d (2D); blocks 0: single steps only
    RingLaunch ppcg2p;          // 3D: the same with the preconditioner (its rows staged: more shared memory)
    RingLaunch ppcg2_32;        // k_ppcg2_ring{2,3}d<PpcgF32>: the FP32 inner PPCG; blocks 0: none
    int stencil_mode = 0;  // 0: the faster kernel per sweep, 1: register pipeline only, 2: ring only
    Loop loops[LOOP_COUNT];
    bool use_graph = true;
};

Fused* fused_of(Chunk* c) { return static_cast<Fused*>(c->fused); }

// FP32-refined form: an inner solve may stop once its sum r^2 is below this fraction of the
// outer target eps (the rounding of the FP32 correction is far below it at that point).
constexpr double kInnerTargetMargin = 0.1;

// After a warm start replaced u (and r = u0 - A u was recomputed): the CG start
// p = z = Mi r (preconditioned) or p = r, and rro = sum r.p -- CGCalcRRO's last part.
__global__ void __launch_bounds__(BLOCK) k_ws_restart(Geom g, Box inner, Fields f, int precond, RedScratch rs,
                                                      double* out)
{
    DDVec<1> acc;
    acc.zero();
    walk(inner, [&](int kk, int jj, int ii) {
        const long i = fidx(g, kk, jj, ii);
        const double r = f.r[i];
        double p = r;
        if (precond) {
            p = f.mi[i] * r;
            f.z[i] = p;
        }
        f.p[i] = p;
        dd_add(acc.v[0], r * p);
    });
    grid_reduce<1>(acc, rs, out);
}

// Back to the plain start after a rejected guess: inner u = u0 (the set-up's u, bit for bit).
__global__ void __launch_bounds__(BLOCK) k_ws_restore(Geom g, Box inner, Fields f)
{
    walk(inner, [&](int kk, int jj, int ii) {
        const long i = fidx(g, kk, jj, ii);
        f.u[i] = f.u0[i];
    });
}

void free_loops(Fused* F)
{
    for (Loop& l : F->loops) {
        if (l.exec) cudaGraphExecDestroy(l.exec);
        if (l.graph) cudaGraphDestroy(l.graph);
        l = Loop();
    }
}

template <class K>
int occupancy(K kernel, int threads)
{
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, 0) != cudaSuccess || n < 1) n = 1;
    return n;
}

#if TEA_DIM == 2
constexpr size_t ppcg2_2d_smem_bytes = (size_t)RWARPS * C2_RQ * C2_NA * Pair2Geom<double>::STRIP * sizeof(double);
#endif

// CG iterations per launch of the while node's body.
constexpr int kCgUnroll = 4;

// PPCG inner steps that run as two-step passes: an even number of pairs, none holding the
// last step (which forms the 2-norm).
// Two-step PPCG passes per outer iteration: every step in pairs when the count is even (the
// last pair also forms the 2-norm), else an even number of pairs and single steps after
// them, so that the single steps find sd in the buffer they expect.
inline int ppcg_pairs(int inner_steps)
{
    int pairs = inner_steps / 2;
    if ((inner_steps & 1) && (pairs & 1)) pairs -= 1;
    return pairs;
}

// Opt a ring kernel into its dynamic shared memory; blocks per SM it then reaches.
template <class K>
int smem_occupancy(K kernel, int bytes, int threads = RWARPS * 32)
{
    TEA_CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, bytes) != cudaSuccess || n < 1) n = 1;
    return n;
}

#if TEA_DIM == 2

// One wave: every resident warp gets one segment of a strip `strip` columns wide, the
// segment length chosen so that the strips' segments fill the resident warps.
RingLaunch ring_launch(const Geom& g, int sms, int occ, int strip, int max_blocks)
{
    const long warps = (long)sms * occ * RWARPS;
    const long per_x = (g.nx + strip - 1) / strip;
    long per_y = std::max<long>(1, warps / per_x);
    RingLaunch L;
    L.rows = (int)std::max<long>(8, (g.ny + per_y - 1) / per_y);
    per_y = (g.ny + L.rows - 1) / L.rows;
    long blocks = std::min<long>((per_x * per_y + RWARPS - 1) / RWARPS, (long)sms * occ);
    L.blocks = (int)std::max<long>(1, std::min<long>(blocks, max_blocks));
    return L;
}

#endif

template <class Op>
struct RingId;
template <>
struct RingId<OpSweepA> {
    static constexpr int value = 0;
};
template <>
struct RingId<OpCheby> {
    static constexpr int value = 1;
};
template <>
struct RingId<OpPPCGInner<false>> {
    static constexpr int value = 2;
};
template <>
struct RingId<OpPPCGInner<true>> {
    static constexpr int value = 3;
};
template <>
struct RingId<OpJacobi> {
    static constexpr int value = 4;
};
template <>
struct RingId<OpJacobiResidual> {
    static constexpr int value = 5;
};
template <>
struct RingId<OpSweepA32> {
    static constexpr int value = 6;
};
template <>
struct RingId<OpOuterResid> {
    static constexpr int value = 7;
};
template <>
struct RingId<OpCheby32> {
    static constexpr int value = 8;
};

#if TEA_DIM == 2
template <class Op>
void setup_ring(Fused* F, const Geom& g, int sms, int max_blocks)
{
    const int occ = smem_occupancy(k_ring2d<Op>, (int)ring_smem_bytes<Op>());
    F->ring[RingId<Op>::value] = ring_launch(g, sms, occ, RingGeomOf<Op>::STRIP, max_blocks);
}
#else
// Grid and z-segment length of k_ring3d: units (x-y tile, z segment) are dealt to the
// resident blocks round-robin; the segment length minimises the waves times the planes a
// unit streams (its own plus about two of pipeline start-up).
RingLaunch ring3_launch(const Geom& g, int sms, int occ, int strip, int ty, int max_blocks)
{
    const long slots = std::max<long>(1, std::min<long>((long)sms * occ, max_blocks));
    const long txy = (long)((g.nx + strip - 1) / strip) * ((g.ny + ty - 1) / ty);
    RingLaunch L;
    long best = -1;
    for (int nseg = 1; nseg <= g.nz; ++nseg) {
        const int len = (g.nz + nseg - 1) / nseg;
        if (nseg > 1 && len == (g.nz + nseg - 2) / (nseg - 1)) continue;  // same length as before
        const long units = txy * ((g.nz + len - 1) / len);
        const long waves = (units + slots - 1) / slots;
        const long cost = waves * (len + 2);
        if (best < 0 || cost < best) {
            best = cost;
            L.rows = len;
            L.blocks = (int)std::min(units, slots);
        }
    }
    return L;
}

// Rows per tile (warps per block) and planes in flight of each sweep's k_ring3d, measured
// on B200 at 512^3 over TY in {2, 4, 6, 8} and RP in {1, 2, 3, 4, 6}.
template <class Op>
struct Ring3Cfg {
    static constexpr int TY = 4, RP = 2;
};
template <bool P>
struct Ring3Cfg<OpPPCGInner<P>> {
    static constexpr int TY = 4, RP = 3;
};
template <>
struct Ring3Cfg<OpJacobi> {
    static constexpr int TY = 8, RP = 2;
};
template <>
struct Ring3Cfg<OpJacobiResidual> {
    static constexpr int TY = 8, RP = 2;
};
template <>
struct Ring3Cfg<OpOuterResid> {
    static constexpr int TY = 8, RP = 2;
};
template <>
struct Ring3Cfg<OpCheby32> {
    static constexpr int TY = 8, RP = 1;
};

template <class Op>
constexpr auto ring3_kernel()
{
    return k_ring3d<Op, Ring3Cfg<Op>::TY, Ring3Cfg<Op>::RP>;
}
template <class Op>
constexpr size_t ring3_bytes()
{
    return ring3_smem_bytes<Op, Ring3Cfg<Op>::TY, Ring3Cfg<Op>::RP>();
}

// Rows per tile and planes in flight of the two-step PPCG pass (3D), measured on B200 at
// 512^3 over (TY, RP) in {(4, 1), (6, 1), (6, 2), (8, 1), (8, 2), (10, 1)}.
#ifndef TEA_PPCG2_TY
#define TEA_PPCG2_TY 8
#endif
#ifndef TEA_PPCG2_RP
#define TEA_PPCG2_RP 2
#endif
#ifndef TEA_PPCG2_RP_PLAIN
#define TEA_PPCG2_RP_PLAIN 1
#endif
// The 3D two-step PPCG pass: TY rows per tile, RP planes in flight with the preconditioner,
// RP_PLAIN without it (whose smaller ring slots then fit two blocks on an SM).
constexpr int PPCG2_TY = TEA_PPCG2_TY, PPCG2_RP = TEA_PPCG2_RP, PPCG2_RP_PLAIN = TEA_PPCG2_RP_PLAIN;

template <class Op>
void setup_ring3(Fused* F, const Geom& g, int sms, int max_blocks)
{
    constexpr int ty = Ring3Cfg<Op>::TY;
    const int occ = smem_occupancy(ring3_kernel<Op>(), (int)ring3_bytes<Op>(), ty * 32);
    F->ring3[RingId<Op>::value] = ring3_launch(g, sms, occ, RingGeomOf<Op>::STRIP, ty, max_blocks);
}
#endif

#if TEA_DIM == 2
// Which 2D sweeps run the shared-memory ring by default (measured on B200 at 4096^2: the
// ring is faster for CG sweep A, the Chebyshev iteration and Jacobi, the register pipeline
// for the PPCG inner step).
template <class Op>
struct RingPreferred {
    static constexpr bool value = false;
};
template <>
struct RingPreferred<OpSweepA> {
    static constexpr bool value = true;
};
template <>
struct RingPreferred<OpCheby> {
    static constexpr bool value = true;
};
template <>
struct RingPreferred<OpSweepA32> {
    static constexpr bool value = true;
};
template <>
struct RingPreferred<OpOuterResid> {
    static constexpr bool value = true;
};
template <>
struct RingPreferred<OpCheby32> {
    static constexpr bool value = true;
};
template <>
struct RingPreferred<OpJacobi> {
    static constexpr bool value = true;
};
template <>
struct RingPreferred<OpJacobiResidual> {
    static constexpr bool value = true;
};
#else
// Every 3D sweep runs the plane ring by default.
template <class Op>
struct RingPreferred {
    static constexpr bool value = true;
};
#endif

// Launch the streaming stencil kernel of Op over the inner domain.
template <class Op>
void stencil(const Fused* F, const FusedArgs& a, cudaStream_t s)
{
#if TEA_DIM == 2
    if (F->stencil_mode == 2 || (F->stencil_mode == 0 && RingPreferred<Op>::value)) {
        const RingLaunch& L = F->ring[RingId<Op>::value];
        FusedArgs ar = a;
        ar.seg_rows = L.rows;
        k_ring2d<Op><<<L.blocks, RWARPS * 32, ring_smem_bytes<Op>(), s>>>(ar);
        return;
    }
#else
    if (F->stencil_mode == 2 || (F->stencil_mode == 0 && RingPreferred<Op>::value)) {
        const RingLaunch& L = F->ring3[RingId<Op>::value];
        FusedArgs ar = a;
        ar.seg_rows = L.rows;
        ring3_kernel<Op>()<<<L.blocks, Ring3Cfg<Op>::TY * 32, ring3_bytes<Op>(), s>>>(ar);
        return;
    }
#endif
    TEA_STENCIL<Op><<<F->stencil_blocks, TEA_STENCIL_BLOCK, 0, s>>>(a);
}

Fused* ensure_fused(Chunk* c, int max_iters)
{
    Fused* F = fused_of(c);
    if (!F) {
        F = new Fused();
        c->fused = F;
        const char* env = std::getenv("TEA_B200_NO_GRAPH");
        F->use_graph = !(env && env[0] == '1');
        TEA_CK(cudaMalloc(&F->d_st, sizeof(SolveState)));
        TEA_CK(cudaMemset(F->d_st, 0, sizeof(SolveState)));
        TEA_CK(cudaHostAlloc(&F->h_st, sizeof(SolveState), cudaHostAllocDefault));
        for (int k = 0; k < 3; ++k) {
            TEA_CK(cudaMalloc(&F->alt[k], c->field_elems * sizeof(double)));
            if (F->alt[k]) TEA_CK(cudaMemset(F->alt[k], 0, c->field_elems * sizeof(double)));
        }
        // The clears ran on the legacy stream, which does not order with the chunk's
        // non-blocking stream: finish them before any kernel there can touch the arrays.
        TEA_CK(cudaDeviceSynchronize());
        const Geom& g = c->g;
        FusedArgs& a = F->base;
        a.g = g;
        a.u[0] = c->f.u;
        a.u[1] = F->alt[0] + kLeadPad;
        a.p[0] = c->f.p;
        a.p[1] = F->alt[1] + kLeadPad;
        a.sd[0] = c->f.sd;
        a.sd[1] = F->alt[2] + kLeadPad;
        a.r = c->f.r;
        a.w = c->f.w;
        a.z = c->f.z;
        a.mi = c->f.mi;
        a.u0 = c->f.u0;
        a.kx = c->f.kx;
        a.ky = c->f.ky;
        a.kz = c->f.kz;
        a.st = F->d_st;
        a.red = c->red;
        a.use_handle = 0;
        a.step = 0;
        a.timing = 0;
        a.r_in_w = 0;
        a.seg_rows = 64;  // every ring launch sets its own
        int sms = 148;
        TEA_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
        if (DIM == 2) {
            a.tiles_x = (g.nx + SBLOCK - 1) / SBLOCK;
            a.tiles_y = (g.ny + SY - 1) / SY;
            a.zseg = 1;
            a.ntiles = (long)a.tiles_x * a.tiles_y;
        } else {
            a.tiles_x = (g.nx + 31) / 32;
            a.tiles_y = (g.ny + TY3 - 1) / TY3;
            const long txy = (long)a.tiles_x * a.tiles_y;
            int zseg = g.nz;
            const long want = 8L * sms * 4;
            while (zseg > 8 && txy * ((g.nz + zseg - 1) / zseg) < want) zseg = (zseg + 1) / 2;
            a.zseg = zseg;
            a.ntiles = txy * ((g.nz + zseg - 1) / zseg);
        }
        const int nthr = (int)(TEA_STENCIL_BLOCK.x * TEA_STENCIL_BLOCK.y);
        int occ = occupancy(TEA_STENCIL<OpSweepA>, nthr);
        occ = std::min(occ, occupancy(TEA_STENCIL<OpCheby>, nthr));
        occ = std::min(occ, occupancy(TEA_STENCIL<OpPPCGInner<true>>, nthr));
        occ = std::min(occ, occupancy(TEA_STENCIL<OpJacobi>, nthr));
        occ = std::min(occ, occupancy(TEA_STENCIL<OpSweepA32>, nthr));
        occ = std::min(occ, occupancy(TEA_STENCIL<OpOuterResid>, nthr));
        occ = std::min(occ, occupancy(TEA_STENCIL<OpCheby32>, nthr));
        F->stencil_blocks = (int)std::min<long>(a.ntiles, (long)sms * occ);
        F->stencil_blocks = std::min(F->stencil_blocks, c->red.max_blocks);
        F->stencil_blocks = std::max(F->stencil_blocks, 1);
        {
            // TEA_B200_STENCIL=pipe|ring forces one kernel family for every sweep (A/B timing).
            const char* kind = getenv("TEA_B200_STENCIL");
            F->stencil_mode = !kind ? 0 : (strcmp(kind, "pipe") == 0 ? 1 : (strcmp(kind, "ring") == 0 ? 2 : 0));
        }
#if TEA_DIM == 3
        if (F->stencil_mode != 1) {
            const int mb = c->red.max_blocks;
            setup_ring3<OpSweepA>(F, g, sms, mb);
            setup_ring3<OpCheby>(F, g, sms, mb);
            setup_ring3<OpPPCGInner<false>>(F, g, sms, mb);
            setup_ring3<OpPPCGInner<true>>(F, g, sms, mb);
            setup_ring3<OpJacobi>(F, g, sms, mb);
            setup_ring3<OpJacobiResidual>(F, g, sms, mb);
            setup_ring3<OpSweepA32>(F, g, sms, mb);
            setup_ring3<OpOuterResid>(F, g, sms, mb);
            setup_ring3<OpCheby32>(F, g, sms, mb);
            const int occ = smem_occupancy(k_ppcg2_ring3d<PpcgF64, PPCG2_TY, PPCG2_RP_PLAIN, false>,
                                           (int)ppcg2_smem_bytes<double, PPCG2_TY, PPCG2_RP_PLAIN, false>(),
                                           PPCG2_TY * 32);
            F->ppcg2 = ring3_launch(g, sms, occ, 30 * RingGeom<double>::VEC, PPCG2_TY - 2, mb);
            const int occp = smem_occupancy(k_ppcg2_ring3d<PpcgF64, PPCG2_TY, PPCG2_RP, true>,
                                            (int)ppcg2_smem_bytes<double, PPCG2_TY, PPCG2_RP, true>(), PPCG2_TY * 32);
            F->ppcg2p = ring3_launch(g, sms, occp, 30 * RingGeom<double>::VEC, PPCG2_TY - 2, mb);
            const int occ32 = smem_occupancy(k_ppcg2_ring3d<PpcgF32, PPCG2_TY, PPCG2_RP_PLAIN, false>,
                                             (int)ppcg2_smem_bytes<float, PPCG2_TY, PPCG2_RP_PLAIN, false>(),
                                             PPCG2_TY * 32);
            F->ppcg2_32 = ring3_launch(g, sms, occ32, 30 * RingGeom<float>::VEC, PPCG2_TY - 2, mb);
        }
#else
        {
            if (F->stencil_mode != 1) {
                const int mb = c->red.max_blocks;
                setup_ring<OpSweepA>(F, g, sms, mb);
                setup_ring<OpCheby>(F, g, sms, mb);
                setup_ring<OpPPCGInner<false>>(F, g, sms, mb);
                setup_ring<OpPPCGInner<true>>(F, g, sms, mb);
                setup_ring<OpJacobi>(F, g, sms, mb);
                setup_ring<OpJacobiResidual>(F, g, sms, mb);
                setup_ring<OpSweepA32>(F, g, sms, mb);
                setup_ring<OpOuterResid>(F, g, sms, mb);
                setup_ring<OpCheby32>(F, g, sms, mb);
                const int occ2 = smem_occupancy(k_cheby2_ring2d<OpCheby>, (int)cheby2_smem_bytes<OpCheby>());
                F->pair = ring_launch(g, sms, occ2, Pair2Geom<double>::OUT, mb);
                const int occ3 =
                    smem_occupancy(k_cheby2_ring2d<OpCheby32>, (int)cheby2_smem_bytes<OpCheby32>());
                F->pair32 = ring_launch(g, sms, occ3, Pair2Geom<float>::OUT, mb);
                // The larger (preconditioned) size last: it stays the kernel's opt-in limit.
                const int occq = smem_occupancy(k_cheby4_ring2d<OpCheby>, (int)cheby4_smem_bytes<OpCheby>(false));
                F->quad = ring_launch(g, sms, occq, SkewGeom<double, 4, C4_RP>::OUT, mb);
                const int occqp = smem_occupancy(k_cheby4_ring2d<OpCheby>, (int)cheby4_smem_bytes<OpCheby>(true));
                F->quadp = ring_launch(g, sms, occqp, SkewGeom<double, 4, C4_RP>::OUT, mb);
                const int occq32 =
                    smem_occupancy(k_cheby4_ring2d<OpCheby32>, (int)cheby4_smem_bytes<OpCheby32>(false));
                F->quad32 = ring_launch(g, sms, occq32, SkewGeom<float, 4, C4_RP>::OUT, mb);
                const int occ4 = smem_occupancy(k_ppcg2_ring2d<PpcgF64>, (int)ppcg2_2d_smem_bytes);
                F->ppcg2 = ring_launch(g, sms, occ4, Pair2Geom<double>::OUT, mb);
                const int occ5 = smem_occupancy(k_ppcg2_ring2d<PpcgF32>, (int)ppcg2_2d_smem_bytes);
                F->ppcg2_32 = ring_launch(g, sms, occ5, Pair2Geom<float>::OUT, mb);
            }
        }
#endif
        F->point_blocks = launch_blocks(c, c->inner.ntiles);
        {
            // Segment walks: at most one segment per warp, and at most one wave of the
            // resident blocks, so that no partial second wave trails the first.
            int occ_pair = occupancy(k_cg_sweep_b, 256);
            occ_pair = std::min(occ_pair, occupancy(k_ppcg_sweep_b, 256));
            occ_pair = std::min(occ_pair, occupancy(k_dc_update, 256));
            const long wave_pair = (long)sms * occ_pair;
            const long warps = make_seg(g).nseg;  // one 64-cell segment per warp at most
            const long blocks = (warps + 7) / 8;
            F->pair_blocks =
                (int)std::max<long>(1, std::min<long>(std::min<long>(blocks, wave_pair), c->red.max_blocks));
            const long wave_quad = (long)sms * occupancy(k_cg32_sweep_b, 256);
            const long qwarps = (long)((g.nx + 127) / 128) * g.ny * g.nz;  // one 128-cell segment per warp
            F->quad_blocks =
                (int)std::max<long>(1, std::min<long>(std::min<long>((qwarps + 7) / 8, wave_quad), c->red.max_blocks));
        }
    }
    if (F->cap < max_iters + 2) {
        free_loops(F);  // the graphs hold the old pointers
        for (double* p : {F->d_cg_alphas, F->d_cg_betas, F->d_ch_alphas, F->d_ch_betas})
            if (p) TEA_CK(cudaFree(p));
        F->cap = max_iters + 2;
        TEA_CK(cudaMalloc(&F->d_cg_alphas, sizeof(double) * F->cap));
        TEA_CK(cudaMalloc(&F->d_cg_betas, sizeof(double) * F->cap));
        TEA_CK(cudaMalloc(&F->d_ch_alphas, sizeof(double) * F->cap));
        TEA_CK(cudaMalloc(&F->d_ch_betas, sizeof(double) * F->cap));
        TEA_CK(cudaMemset(F->d_ch_alphas, 0, sizeof(double) * F->cap));
        TEA_CK(cudaMemset(F->d_ch_betas, 0, sizeof(double) * F->cap));
        TEA_CK(cudaDeviceSynchronize());  // legacy-stream clears before the chunk's stream uses them
        F->base.cg_alphas = F->d_cg_alphas;
        F->base.cg_betas = F->d_cg_betas;
        F->base.ch_alphas = F->d_ch_alphas;
        F->base.ch_betas = F->d_ch_betas;
    }
    return F;
}

// The FP32 arrays of the defect-correction form, allocated on first use (same pitched
// layout as the FP64 fields, float elements).
bool ensure_fp32(Chunk* c, Fused* F)
{
    if (F->alloc32[0]) return true;
    const size_t bytes = c->field_elems * sizeof(float);
    for (int k = 0; k < 10; ++k) {
        if (k == 2 && DIM != 3) continue;  // Kz (3D only)
        TEA_CK(cudaMalloc(&F->alloc32[k], bytes));
        if (!F->alloc32[k]) return false;
        TEA_CK(cudaMemset(F->alloc32[k], 0, bytes));
    }
    TEA_CK(cudaDeviceSynchronize());  // legacy-stream clears before the chunk's stream uses them
    free_loops(F);  // graphs captured before hold null FP32 pointers
    FusedArgs& a = F->base;
    a.kx32 = F->alloc32[0] + kLeadPad;
    a.ky32 = F->alloc32[1] + kLeadPad;
    a.kz32 = DIM == 3 ? F->alloc32[2] + kLeadPad : nullptr;
    a.r32 = F->alloc32[3] + kLeadPad;
    a.w32 = F->alloc32[4] + kLeadPad;
    a.d32 = F->alloc32[5] + kLeadPad;
    a.p32[0] = F->alloc32[6] + kLeadPad;
    a.p32[1] = F->alloc32[7] + kLeadPad;
    a.dc32[0] = a.d32;
    a.dc32[1] = a.w32;
    a.sd32[0] = F->alloc32[8] + kLeadPad;
    a.sd32[1] = F->alloc32[9] + kLeadPad;
    return true;
}

#if TEA_DIM == 3
// The 3D two-step PPCG pass, in the form of the solve's preconditioner.
void launch_ppcg2_3d(Fused* F, const FusedArgs& a, bool precond, cudaStream_t s)
{
    FusedArgs ak = a;
    if (precond) {
        ak.seg_rows = F->ppcg2p.rows;
        k_ppcg2_ring3d<PpcgF64, PPCG2_TY, PPCG2_RP, true>
            <<<F->ppcg2p.blocks, PPCG2_TY * 32, ppcg2_smem_bytes<double, PPCG2_TY, PPCG2_RP, true>(), s>>>(ak);
    } else {
        ak.seg_rows = F->ppcg2.rows;
        k_ppcg2_ring3d<PpcgF64, PPCG2_TY, PPCG2_RP_PLAIN, false>
            <<<F->ppcg2.blocks, PPCG2_TY * 32, ppcg2_smem_bytes<double, PPCG2_TY, PPCG2_RP_PLAIN, false>(), s>>>(ak);
    }
}
#endif

#if TEA_DIM == 2

// The four-iteration FP64 Chebyshev pass, with the launch of the solve's preconditioner
// setting (with mi staged it needs more shared memory per warp).
void launch_cheby4(Fused* F, const FusedArgs& a, bool precond, cudaStream_t s)
{
    const RingLaunch& L = precond ? F->quadp : F->quad;
    FusedArgs ap = a;
    ap.seg_rows = L.rows;
    k_cheby4_ring2d<OpCheby><<<L.blocks, RWARPS * 32, cheby4_smem_bytes<OpCheby>(precond), s>>>(ap);
}
#endif

// Enqueue one iteration of loop `kind` on the chunk's stream.
void enqueue_body(Chunk* c, Fused* F, int kind, int inner_steps, const FusedArgs& a)
{
    cudaStream_t s = c->stream;
    switch (kind) {
    case LOOP_CG:
        // Unrolled: the while node relaunches its body once per kCgUnroll iterations.  Once
        // an iteration ends the loop (cont = 0), the kernels of the later copies return at
        // once, so the iterations run are exactly those of the rolled loop.
        for (int k = 0; k < kCgUnroll; ++k) {
            stencil<OpSweepA>(F, a, s);
            k_cg_sweep_b<<<F->pair_blocks, 256, 0, s>>>(a);
        }
        break;
    case LOOP_CHEBY:
#if TEA_DIM == 2
        if (F->quad.blocks > 0) {
            launch_cheby4(F, a, F->h_st->precond != 0, s);
            break;
        }
        if (F->pair.blocks > 0) {
            FusedArgs ap = a;
            ap.seg_rows = F->pair.rows;
            k_cheby2_ring2d<OpCheby><<<F->pair.blocks, RWARPS * 32, cheby2_smem_bytes<OpCheby>(), s>>>(ap);
            break;
        }
#endif
        stencil<OpCheby>(F, a, s);
        break;
    case LOOP_CHEBY32:
#if TEA_DIM == 2
        if (F->quad32.blocks > 0) {
            FusedArgs ap = a;
            ap.seg_rows = F->quad32.rows;
            k_cheby4_ring2d<OpCheby32>
                <<<F->quad32.blocks, RWARPS * 32, cheby4_smem_bytes<OpCheby32>(false), s>>>(ap);
            break;
        }
        if (F->pair32.blocks > 0) {
            FusedArgs ap = a;
            ap.seg_rows = F->pair32.rows;
            k_cheby2_ring2d<OpCheby32>
                <<<F->pair32.blocks, RWARPS * 32, cheby2_smem_bytes<OpCheby32>(), s>>>(ap);
            break;
        }
#endif
        stencil<OpCheby32>(F, a, s);
        break;
    case LOOP_PPCG: {
        stencil<OpSweepA>(F, a, s);
        // r alternates between r and w over the pairs; with an odd number of pairs sweep B
        // leaves r in w, so that the last pair writes it back into r.
        const int pairs = F->ppcg2.blocks > 0 ? ppcg_pairs(inner_steps) : 0;
        FusedArgs ab = a;
        ab.r_in_w = pairs & 1;
        k_ppcg_sweep_b<<<F->pair_blocks, 256, 0, s>>>(ab);
        int k0 = 1;
        for (int m = 1; m <= pairs; ++m, k0 += 2) {
            FusedArgs ak = ab;
            ak.step = k0;
            ak.seg_rows = F->ppcg2.rows;
#if TEA_DIM == 2
            k_ppcg2_ring2d<PpcgF64><<<F->ppcg2.blocks, RWARPS * 32, ppcg2_2d_smem_bytes, s>>>(ak);
#else
            launch_ppcg2_3d(F, ak, F->h_st->precond != 0, s);
#endif
        }
        for (int k = k0; k <= inner_steps; ++k) {
            FusedArgs ak = a;
            ak.step = k;
            if (k < inner_steps) stencil<OpPPCGInner<false>>(F, ak, s);
            else stencil<OpPPCGInner<true>>(F, ak, s);
        }
        break;
    }
    case LOOP_JACOBI:
        stencil<OpJacobi>(F, a, s);
        stencil<OpJacobiResidual>(F, a, s);
        break;
    case LOOP_CG32:
        stencil<OpSweepA32>(F, a, s);
        k_cg32_sweep_b<<<F->quad_blocks, 256, 0, s>>>(a);
        break;
    case LOOP_PPCG32: {
        // One FP32 inner PPCG iteration (an even number of inner steps, all in pairs):
        // p = r + beta p and w = A p with p.w, then d += alpha p, r -= alpha w, sd = r / theta,
        // then the inner steps; the last pair forms r.r and ends the iteration.
        stencil<OpSweepA32>(F, a, s);
        const int pairs = inner_steps / 2;
        FusedArgs ab = a;
        ab.r_in_w = pairs & 1;
        k_ppcg32_sweep_b<<<F->quad_blocks, 256, 0, s>>>(ab);
        for (int m = 1, k0 = 1; m <= pairs; ++m, k0 += 2) {
            FusedArgs ak = ab;
            ak.step = k0;
            ak.seg_rows = F->ppcg2_32.rows;
#if TEA_DIM == 2
            k_ppcg2_ring2d<PpcgF32><<<F->ppcg2_32.blocks, RWARPS * 32, ppcg2_2d_smem_bytes, s>>>(ak);
#else
            k_ppcg2_ring3d<PpcgF32, PPCG2_TY, PPCG2_RP_PLAIN, false><<<F->ppcg2_32.blocks, PPCG2_TY * 32,
                                                                      ppcg2_smem_bytes<float, PPCG2_TY, PPCG2_RP_PLAIN,
                                                                                       false>(),
                                                                      s>>>(ak);
#endif
        }
        break;
    }
    }
}

// Build (once per chunk, loop kind and inner-step count) a graph holding a while-node
// whose body is one iteration.
bool build_loop(Chunk* c, Fused* F, int kind, int inner_steps)
{
    Loop& L = F->loops[kind];
    // The Chebyshev and PPCG bodies' launches depend on the preconditioner (their shared memory).
    const int key = kind == LOOP_PPCG ? 2 * inner_steps + (F->h_st->precond ? 1 : 0)
                                      : (kind == LOOP_PPCG32 ? inner_steps
                                                             : (kind == LOOP_CHEBY ? F->h_st->precond : 0));
    if (L.exec && L.key == key) return true;
    if (L.exec) cudaGraphExecDestroy(L.exec);
    if (L.graph) cudaGraphDestroy(L.graph);
    L = Loop();
    cudaGraph_t graph = nullptr;
    if (cudaGraphCreate(&graph, 0) != cudaSuccess) return false;
    cudaGraphConditionalHandle handle;
    cudaError_t e = cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault);
    if (e != cudaSuccess) {
        set_status(TEA_ERR_CUDA, "cudaGraphConditionalHandleCreate: %s", cudaGetErrorString(e));
        cudaGraphDestroy(graph);
        return false;
    }
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = handle;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    e = cudaGraphAddNode(&node, graph, nullptr, 0, &cp);
    if (e != cudaSuccess) {
        set_status(TEA_ERR_CUDA, "cudaGraphAddNode(while): %s", cudaGetErrorString(e));
        cudaGraphDestroy(graph);
        return false;
    }
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    FusedArgs a = F->base;
    a.handle = handle;
    a.use_handle = 1;
    TEA_CK(cudaStreamBeginCaptureToGraph(c->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    enqueue_body(c, F, kind, inner_steps, a);
    cudaGraph_t captured = nullptr;
    TEA_CK(cudaStreamEndCapture(c->stream, &captured));
    e = cudaGraphInstantiate(&L.exec, graph, 0);
    if (e != cudaSuccess) {
        set_status(TEA_ERR_CUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(e));
        cudaGraphDestroy(graph);
        L = Loop();
        return false;
    }
    L.graph = graph;
    L.key = key;
    return true;
}

// The host record is pinned and the host rewrites it right after most pushes, so the copy
// has read it before this returns.
void push_state(Chunk* c, Fused* F)
{
    TEA_CK(cudaMemcpyAsync(F->d_st, F->h_st, sizeof(SolveState), cudaMemcpyHostToDevice, c->stream));
    c->h2d_bytes += sizeof(SolveState);
    sync(c);
}

void pull_state(Chunk* c, Fused* F)
{
    TEA_CK(cudaMemcpyAsync(F->h_st, F->d_st, sizeof(SolveState), cudaMemcpyDeviceToHost, c->stream));
    c->d2h_bytes += sizeof(SolveState);
    sync(c);
}

// Run loop `kind` from the current state until its exit; the host state is refreshed.
void run_loop(Chunk* c, Fused* F, int kind, int inner_steps)
{
    F->h_st->cont = 1;  // the body runs at least once (the while node's default)
    push_state(c, F);
    if (F->use_graph && build_loop(c, F, kind, inner_steps)) {
        TEA_CK(cudaGraphLaunch(F->loops[kind].exec, c->stream));
        pull_state(c, F);
        return;
    }
    // Without graphs: one iteration per launch sequence, the exit flag read back each time.
    FusedArgs a = F->base;
    for (;;) {
        enqueue_body(c, F, kind, inner_steps, a);
        pull_state(c, F);
        if (!F->h_st->cont || status_store().status == TEA_ERR_CUDA) break;
    }
}

// Host mirror of end_iteration() for the iterations run by per-call kernels.
void end_iteration_host(SolveState& s, int phase)
{
    const int n = s.n;
    int cont = 1, reason = EXIT_NONE;
    if (std::fabs(s.error) < s.eps) {
        cont = 0;
        reason = EXIT_CONVERGED;
    } else if (n + 1 > s.max_iters) {
        cont = 0;
        reason = EXIT_MAXITER;
    } else if (s.solver == SOLVER_CHEBY || s.solver == SOLVER_PPCG) {
        const bool sw = s.errswitch ? (s.cheby_calc_steps > 0) || ((s.error <= s.epslim) && (n + 1 >= 20))
                                    : (n + 1 >= s.presteps) && (s.error <= 1.0);
        if ((phase == PHASE_CG) == sw) {
            cont = 0;
            reason = EXIT_PHASE;
        }
    }
    if (reason != EXIT_CONVERGED) s.n = n + 1;
    s.cont = cont;
    s.exit_reason = reason;
}

bool switch_check_host(const SolveState& s, int n)
{
    if (s.errswitch) return (s.cheby_calc_steps > 0) || ((s.error <= s.epslim) && (n >= 20));
    return (n >= s.presteps) && (s.error <= 1.0);
}

const int kAllExternal[6] = {-1, -1, -1, -1, -1, -1};

void halo(Chunk* c, std::initializer_list<int> ids, int depth)
{
    int fields[6] = {0, 0, 0, 0, 0, 0};
    for (int id : ids) fields[id - 1] = 1;
    update_halo(c, kAllExternal, fields, depth);
}

// Bring u and p to the state the per-call kernels expect: pending updates applied,
// current values in the canonical buffers, the depth-1 halo of u reflected and that of
// p reflected when the reference's halo field list holds p at this point (it does not
// in Chebyshev mode before a CG iteration has run, tealeaf_2d/tea_solve.f90:203-204).
void canonicalize(Chunk* c, Fused* F, bool refresh_p = true)
{
    SolveState& s = *F->h_st;
    FusedArgs a = F->base;
    if (s.pending_p || s.pending_u) {
        push_state(c, F);
        k_flush<<<F->point_blocks, dim3(TILE_X, TILE_Y), 0, c->stream>>>(a, c->inner);
        s.pending_p = 0;
        s.pending_u = 0;
    }
    const size_t bytes = c->field_elems * sizeof(double);
    if (s.par_p) {
        TEA_CK(cudaMemcpyAsync(c->alloc[F_P], F->alt[1], bytes, cudaMemcpyDeviceToDevice, c->stream));
        s.par_p = 0;
    }
    if (s.par_u) {
        TEA_CK(cudaMemcpyAsync(c->alloc[F_U], F->alt[0], bytes, cudaMemcpyDeviceToDevice, c->stream));
        s.par_u = 0;
    }
    push_state(c, F);
    if (refresh_p) halo(c, {4, 5}, 1);
    else halo(c, {4}, 1);
}

}  // namespace

void destroy_fused(Chunk* c)
{
    Fused* F = fused_of(c);
    if (!F) return;
    free_loops(F);
    for (double* p : {F->d_cg_alphas, F->d_cg_betas, F->d_ch_alphas, F->d_ch_betas})
        if (p) cudaFree(p);
    for (double* p : F->alt)
        if (p) cudaFree(p);
    for (float* p : F->alloc32)
        if (p) cudaFree(p);
    if (F->d_st) cudaFree(F->d_st);
    if (F->h_st) cudaFreeHost(F->h_st);
    delete F;
    c->fused = nullptr;
}

}  // namespace tea

using namespace tea;

TEA_EXPORT void ext_tea_leaf_solve_(const int* chunk, const tea_solve_params* P, tea_solve_result* R)
{
    if (R) std::memset(R, 0, sizeof(*R));
    Chunk* c = get_chunk(chunk);
    if (!c || !P || !R) return;
    const int solver = P->solver;
    if (solver < TEA_SOLVER_JACOBI || solver > TEA_SOLVER_PPCG || P->max_iters < 1 ||
        (solver == TEA_SOLVER_PPCG && P->ppcg_inner_steps < 1) ||
        (P->precision != TEA_PRECISION_FP64 && P->precision != TEA_PRECISION_FP32_REFINED)) {
        set_status(TEA_ERR_BAD_ARGUMENT, "ext_tea_leaf_solve_: invalid parameters");
        R->status = TEA_ERR_BAD_ARGUMENT;
        return;
    }
    Fused* F = ensure_fused(c, P->max_iters);
    const bool cg_like = solver != TEA_SOLVER_JACOBI;
    int coefficient = P->coefficient, precond = P->preconditioner ? 1 : 0;
    double dt = P->dt;

    // INIT, tealeaf_2d/tea_solve.f90:79-164.
    halo(c, {3, 1}, 2);
    double rro = 0.0;
    if (cg_like) {
        ext_cg_solver_init_(chunk, &coefficient, &precond, &dt, &rro);
        halo(c, {4, 5}, 1);
    } else {
        ext_jacobi_kernel_init_(chunk, &coefficient, &dt);
    }
    ext_solver_copy_u_(chunk);
    double eps = P->eps;
    if (P->eps_rel > 0.0) {
        double bb = 0.0;
        int zero = 0;
        ext_calculate_2norm_(chunk, &bb, &zero);
        eps = P->eps_rel * P->eps_rel * bb;
    }
    // Learned warm start (a network attached with tea_ws_attach_): keep u = u0 + du when its
    // FP64 residual is smaller than that of u = u0, and restart CG from it.  After three
    // rejected guesses in a row the prediction is skipped for 4 timesteps, then 8, 16 and
    // at most 32 before the next try; an accepted guess ends the back-off.
    int ws_used = 0;
    double ws_r0_plain = 0.0, ws_r0_guess = 0.0;
    const bool ws_try = c->ws && cg_like && c->ws_skip == 0;
    if (c->ws && cg_like && c->ws_skip > 0) --c->ws_skip;
    if (ws_try) {
        int one = 1;
        ext_calculate_2norm_(chunk, &ws_r0_plain, &one);  // r = u0 - A u0 after the set-up
        if (ws_predict_into(c, c->f.u)) {
            // The residual reads u's halo: reflect the guess first.
            halo(c, {4}, 1);
            ext_calculate_residual_(chunk);
            ext_calculate_2norm_(chunk, &ws_r0_guess, &one);
            if (ws_r0_guess < ws_r0_plain) {
                k_ws_restart<<<launch_blocks(c, c->inner.ntiles), dim3(TILE_X, TILE_Y), 0, c->stream>>>(
                    c->g, c->inner, c->f, precond, c->red, c->d_out);
                sync(c);
                rro = ((volatile double*)c->h_out)[0];
                c->d2h_bytes += sizeof(double);
                ws_used = 1;
                c->ws_reject_streak = 0;
                halo(c, {5}, 1);
            } else {
                if (++c->ws_reject_streak >= 3) c->ws_skip = 4 << std::min(c->ws_reject_streak - 3, 3);
                // The set-up's state: inner u = u0 with its reflected halo, r = u0 - A u
                // (the same operations as the set-up's r = u - A u), p and rro untouched.
                k_ws_restore<<<launch_blocks(c, c->inner.ntiles), dim3(TILE_X, TILE_Y), 0, c->stream>>>(
                    c->g, c->inner, c->f);
                halo(c, {4}, 1);
                ext_calculate_residual_(chunk);
            }
        }
    }
    // The second buffers start as copies, so halos the loops never write match u and p.
    const size_t bytes = c->field_elems * sizeof(double);
    TEA_CK(cudaMemcpyAsync(F->alt[0], c->alloc[F_U], bytes, cudaMemcpyDeviceToDevice, c->stream));
    TEA_CK(cudaMemcpyAsync(F->alt[1], c->alloc[F_P], bytes, cudaMemcpyDeviceToDevice, c->stream));

    SolveState& s = *F->h_st;
    std::memset(&s, 0, sizeof(s));
    s.rro = rro;
    s.error = 1e10;
    s.eps = eps;
    s.epslim = P->ch_cg_epslim;
    s.n = 1;
    s.cont = 1;
    s.solver = solver;
    s.precond = precond;
    s.max_iters = P->max_iters;
    s.presteps = P->ch_cg_presteps;
    s.errswitch = P->ch_cg_errswitch ? 1 : 0;
    s.inner_steps = P->ppcg_inner_steps;
    const bool cheby = solver == TEA_SOLVER_CHEBYSHEV, ppcg = solver == TEA_SOLVER_PPCG;
    int switch_step = 0, cg_steps = 0;
    double eigmin = 0.0, eigmax = 0.0;
    // Whether the reference's update_halo field list currently includes p (FIELD_P): true
    // from the CG set-up, false after the Chebyshev switch until a CG iteration runs.
    bool p_halo_fresh = true;

    int corrections = 0;
    int last_inner_mode = 0;  // FP32-refined: inner solver of the last correction kept
    if (P->precision == TEA_PRECISION_FP32_REFINED) {
        // Defect correction: FP64 outer residual, update and convergence test; FP32 inner
        // solves.  CG and Jacobi decks: every inner solve is CG.  Chebyshev and PPCG decks:
        // the first inner solve is CG, whose scalars give the Lanczos eigenvalue bounds
        // (computed in FP64 on the host), and the following ones are Chebyshev (PPCG decks
        // with an even number of inner steps: PPCG with the deck's inner steps) --
        // the plain solve's CG-then-Chebyshev/PPCG order, with the spectrum taken from a CG
        // run long enough to resolve it.
        if (!ensure_fp32(c, F)) {
            R->status = TEA_ERR_CUDA;
            return;
        }
        FusedArgs a = F->base;
        k_coef_to_fp32<<<c->grid_blocks, 256, 0, c->stream>>>(a);
        const double tol = P->inner_tol > 0.0 ? P->inner_tol : 1e-4;
        // Chebyshev decks: the first correction's inner CG also estimates the spectrum.
        const bool want_cheby = cheby || ppcg;
        int inner_mode = 0;  // the inner solve: 0 CG, 1 Chebyshev, 2 PPCG
        const bool ppcg_inner = ppcg && P->inner_solver == TEA_INNER_DECK && P->ppcg_inner_steps >= 2 &&
                                P->ppcg_inner_steps % 2 == 0 && F->ppcg2_32.blocks > 0;
        int total_inner = 0, presteps_done = 0, cg_inner = 0;
        bool converged = false;
        for (int guard = 0; !converged && guard < P->max_iters + 2; ++guard) {
            if (status_store().status == TEA_ERR_CUDA) break;
            push_state(c, F);
            stencil<OpOuterResid>(F, a, c->stream);
            pull_state(c, F);
            if (std::fabs(s.error) < eps || s.nonfinite) {
                s.exit_reason = EXIT_CONVERGED;
                break;
            }
            const int used = presteps_done + total_inner;
            if (used >= P->max_iters) {
                s.exit_reason = EXIT_MAXITER;
                break;
            }
            const int remaining = P->max_iters - used;
            s.inner_max = P->inner_max_iters > 0 ? std::min(P->inner_max_iters, remaining) : remaining;
            // The inner solve reduces the correction's residual by tol, or stops sooner once
            // the outer target is met with a margin (sum r^2 at a tenth of eps): the last
            // correction needs only the reduction that is left.
            s.tol2 = std::max(tol * tol * s.rro, kInnerTargetMargin * eps);
            // The first correction of a Chebyshev or PPCG deck is the CG whose scalars give the
            // eigenvalue bounds: it ends where the plain solve switches (error <= 1 after the
            // presteps, or <= tl_ch_cg_epslim after 20 iterations with tl_ch_cg_errswitch,
            // tealeaf_2d/tea_solve.f90:172-179), whose bounds carry the plain solve's own
            // Chebyshev or PPCG phase, or at the inner tolerance if that comes first.
            const bool first_cg = want_cheby && inner_mode == 0 && corrections == 0;
            s.switch_err = first_cg ? (P->ch_cg_errswitch ? P->ch_cg_epslim : 1.0) : 0.0;
            s.switch_min = P->ch_cg_errswitch ? 20 : P->ch_cg_presteps;
            s.n_inner = inner_mode == 1 ? 1 : 0;
            s.cont = 1;
            s.inner_diverged = 0;
            run_loop(c, F, inner_mode == 1 ? LOOP_CHEBY32 : (inner_mode == 2 ? LOOP_PPCG32 : LOOP_CG32),
                     P->ppcg_inner_steps);
            total_inner += s.n_inner;
            if (inner_mode == 0) cg_inner += s.n_inner;
            if (s.inner_diverged) {
                // The estimated spectrum missed part of it: drop this correction and solve
                // the remaining ones with CG.
                inner_mode = 0;
                s.inner_cheby = 0;
                continue;
            }
            k_dc_update<<<F->pair_blocks, 256, 0, c->stream>>>(a);
            last_inner_mode = inner_mode;
            s.pending_p = 0;
            s.pending_u = 0;
            ++corrections;
            if (want_cheby && corrections == 1 && s.n_inner >= 2) {
                // Lanczos estimate (FP64, host) from the inner CG's scalars; the bounds are
                // widened by 0.95 / 1.05 as the reference widens its own.
                const int n = s.n_inner;
                std::vector<double> ca(n + 1, 0.0), cb(n + 1, 0.0);
                TEA_CK(cudaMemcpyAsync(ca.data(), F->d_cg_alphas, sizeof(double) * (n + 1), cudaMemcpyDeviceToHost,
                                       c->stream));
                TEA_CK(cudaMemcpyAsync(cb.data(), F->d_cg_betas, sizeof(double) * (n + 1), cudaMemcpyDeviceToHost,
                                       c->stream));
                sync(c);
                c->d2h_bytes += 2 * sizeof(double) * (long long)(n + 1);
                if (tea_tridiag_extremes(ca.data() + 1, cb.data() + 1, n, &eigmin, &eigmax) == 0 && eigmin > 0.0 &&
                    eigmax > eigmin) {
                    eigmin = eigmin * kEigMinScale;
                    eigmax = eigmax * kEigMaxScale;
                    const int ncoef = std::min(P->max_iters + 1, F->cap);
                    std::vector<double> ch_a(ncoef, 0.0), ch_b(ncoef, 0.0);
                    double theta = 0.0;
                    tea_calc_ch_coefs(ch_a.data(), ch_b.data(), eigmin, eigmax, &theta, ncoef);
                    TEA_CK(cudaMemcpyAsync(F->d_ch_alphas, ch_a.data(), sizeof(double) * ncoef,
                                           cudaMemcpyHostToDevice, c->stream));
                    TEA_CK(cudaMemcpyAsync(F->d_ch_betas, ch_b.data(), sizeof(double) * ncoef, cudaMemcpyHostToDevice,
                                           c->stream));
                    c->h2d_bytes += 2 * sizeof(double) * (long long)ncoef;
                    const double rk = std::sqrt(eigmax / eigmin);
                    const double rho = (rk - 1.0) / (rk + 1.0);
                    s.theta = theta;
                    s.cheby_rho2 = rho * rho;
                    inner_mode = ppcg_inner ? 2 : 1;
                    s.inner_cheby = inner_mode;
                    switch_step = n + 1;
                }
            }
        }
        if (converged) s.exit_reason = EXIT_CONVERGED;
        cg_steps = presteps_done + cg_inner;
        s.cheby_calc_steps = total_inner - cg_inner + 1;
        s.n = presteps_done + total_inner + 1;
        s.pending_p = s.pending_u = 0;
        s.par_p = 0;
        s.par_u = 0;
        s.inner_cheby = 0;
        push_state(c, F);
    } else if (!cg_like) {
        run_loop(c, F, LOOP_JACOBI, 0);
    } else {
        std::vector<double> ch_alphas, ch_betas;
        double theta = 0.0, cn = 0.0;
        int max_cheby_iters = 0;
        for (int guard = 0; guard < 4 * P->max_iters + 8; ++guard) {
            if (status_store().status == TEA_ERR_CUDA) break;
            const int n = s.n;
            if ((cheby || ppcg) && switch_check_host(s, n)) {
                if (s.cheby_calc_steps == 0) {
                    // The switch, tealeaf_2d/tea_solve.f90:184-223, on the host.
                    canonicalize(c, F);
                    cg_steps = n - 1;
                    std::vector<double> ca(n + 1, 0.0), cb(n + 1, 0.0);
                    TEA_CK(cudaMemcpyAsync(ca.data(), F->d_cg_alphas, sizeof(double) * (n + 1),
                                           cudaMemcpyDeviceToHost, c->stream));
                    TEA_CK(cudaMemcpyAsync(cb.data(), F->d_cg_betas, sizeof(double) * (n + 1),
                                           cudaMemcpyDeviceToHost, c->stream));
                    sync(c);
                    c->d2h_bytes += 2 * sizeof(double) * (long long)(n + 1);
                    max_cheby_iters = P->max_iters - n + 2;
                    s.rro = s.error;
                    int info = tea_calc_eigenvalues(ca.data() + 1, cb.data() + 1, n - 1, &eigmin, &eigmax);
                    if (info != 0) {
                        set_status(TEA_ERR_EIGEN, "tea_leaf: Error in calculating eigenvalues");
                        R->status = TEA_ERR_EIGEN;
                        return;
                    }
                    eigmin = eigmin * kEigMinScale;
                    eigmax = eigmax * kEigMaxScale;
                    const int ncoef = std::max(max_cheby_iters, P->ppcg_inner_steps) + 1;
                    ch_alphas.assign(ncoef, 0.0);
                    ch_betas.assign(ncoef, 0.0);
                    tea_calc_ch_coefs(ch_alphas.data(), ch_betas.data(), eigmin, eigmax, &theta,
                                      cheby ? max_cheby_iters : P->ppcg_inner_steps);
                    cn = eigmax / eigmin;
                    const int nup = std::min<int>((int)ch_alphas.size(), F->cap);
                    TEA_CK(cudaMemcpyAsync(F->d_ch_alphas, ch_alphas.data(), sizeof(double) * nup,
                                           cudaMemcpyHostToDevice, c->stream));
                    TEA_CK(cudaMemcpyAsync(F->d_ch_betas, ch_betas.data(), sizeof(double) * nup,
                                           cudaMemcpyHostToDevice, c->stream));
                    c->h2d_bytes += 2 * sizeof(double) * (long long)nup;
                    switch_step = n;
                    if (cheby) {
                        // tea_leaf_cheby_first_step, tealeaf_2d/tea_solve.f90:658-750.
                        double bb = 0.0, err = 0.0;
                        int zero = 0, one = 1;
                        ext_calculate_2norm_(chunk, &bb, &zero);
                        ext_cheby_solver_init_(chunk, ch_alphas.data(), ch_betas.data(), &theta, &precond,
                                               &max_cheby_iters);
                        halo(c, {4}, 1);
                        ext_cheby_solver_iterate_(chunk, &max_cheby_iters);
                        ext_calculate_2norm_(chunk, &err, &one);
                        s.error = err;
                        s.est_itc = tea_cheby_est_itc(bb, err, cn);
                        s.cheby_calc_steps = 2;
                        halo(c, {4}, 1);
                        p_halo_fresh = false;
                        end_iteration_host(s, PHASE_CHEBY);
                    } else {
                        // First PPCG outer iteration, tealeaf_2d/tea_solve.f90:276-375.
                        s.cheby_calc_steps = 1;
                        ext_ppcg_init_(chunk, ch_alphas.data(), ch_betas.data(), &theta, &max_cheby_iters);
                        ext_calculate_residual_(chunk);
                        halo(c, {4, 5}, 1);
                        double pw = 0.0, rrn = 0.0;
                        ext_cg_calc_w_(chunk, &pw);
                        double alpha = s.rro / pw;
                        ext_cg_calc_ur_(chunk, &alpha, &rrn);
                        ext_ppcg_init_sd_(chunk);
                        for (int k = 1; k <= P->ppcg_inner_steps; ++k) {
                            halo(c, {6}, 1);
                            ext_ppcg_inner_(chunk, &k);
                        }
                        int one = 1;
                        ext_calculate_2norm_(chunk, &rrn, &one);
                        double beta = rrn / s.rro;
                        ext_cg_calc_p_(chunk, &beta);
                        s.error = rrn;
                        s.rro = rrn;
                        s.theta = theta;
                        s.cheby_calc_steps = 2;
                        halo(c, {4, 5}, 1);
                        end_iteration_host(s, PHASE_PPCG);
                    }
                    // Fresh copies for the second buffers (halos as in the canonical ones).
                    TEA_CK(cudaMemcpyAsync(F->alt[0], c->alloc[F_U], bytes, cudaMemcpyDeviceToDevice, c->stream));
                    TEA_CK(cudaMemcpyAsync(F->alt[1], c->alloc[F_P], bytes, cudaMemcpyDeviceToDevice, c->stream));
                    if (s.exit_reason == EXIT_CONVERGED || s.exit_reason == EXIT_MAXITER) break;
                    continue;
                }
                if (cheby) {
                    // The Chebyshev loop may leave p in the second buffer; both start with the
                    // same contents, so the halo (never written in this phase) agrees.
                    TEA_CK(cudaMemcpyAsync(F->alt[1], c->alloc[F_P], bytes, cudaMemcpyDeviceToDevice, c->stream));
                }
                run_loop(c, F, cheby ? LOOP_CHEBY : LOOP_PPCG, P->ppcg_inner_steps);
            } else if (!p_halo_fresh) {
                // A CG iteration in Chebyshev mode (the error rose above 1 after the switch):
                // its ext_cg_calc_w_ reads the halo of p as last refreshed before the switch,
                // so it runs through the per-call kernels, which read halos from memory.
                double pw = 0.0, rrn = 0.0;
                ext_cg_calc_w_(chunk, &pw);
                s.alpha = s.rro / pw;
                ext_cg_calc_ur_(chunk, &s.alpha, &rrn);
                s.beta = rrn / s.rro;
                ext_cg_calc_p_(chunk, &s.beta);
                s.error = rrn;
                s.rro = rrn;
                p_halo_fresh = true;
                halo(c, {4, 5}, 1);
                end_iteration_host(s, PHASE_CG);
                push_state(c, F);
                if (s.exit_reason == EXIT_CONVERGED || s.exit_reason == EXIT_MAXITER) break;
                continue;
            } else {
                run_loop(c, F, LOOP_CG, 0);
            }
            if (s.exit_reason != EXIT_PHASE) break;
            canonicalize(c, F, p_halo_fresh);
        }
    }
    canonicalize(c, F);
    if (s.nonfinite) set_status(TEA_ERR_NONFINITE, "ext_tea_leaf_solve_: non-finite value in a reduction");
    double exact_error = 0.0;
    if (P->check_result) {
        int one = 1;
        ext_calculate_residual_(chunk);
        ext_calculate_2norm_(chunk, &exact_error, &one);
    }
    ext_solver_finalise_(chunk);
    halo(c, {3}, 1);
    sync(c);
    R->iterations = s.n - 1;
    R->status = status_store().status;
    R->cg_steps = (switch_step || P->precision == TEA_PRECISION_FP32_REFINED) ? cg_steps : s.n - 1;
    R->cheby_steps = s.cheby_calc_steps > 0 ? s.cheby_calc_steps - 1 : 0;
    R->switch_step = switch_step;
    R->est_itc = s.est_itc;
    R->error = s.error;
    R->exact_error = exact_error;
    R->eps_used = eps;
    R->eigmin = eigmin;
    R->eigmax = eigmax;
    R->corrections = corrections;
    R->inner_solver = last_inner_mode;
    R->warm_start_used = ws_used;
    R->warm_r0_plain = ws_r0_plain;
    R->warm_r0_guess = ws_r0_guess;
}

// Measurement hook: `reps` back-to-back launches of one fused kernel on the chunk's
// stream between two CUDA events, on the chunk's current fields (their values change).
// kernel: 1 PPCG inner step, 2 CG/PPCG sweep A, 3 Chebyshev iteration, 4 Jacobi sweep,
// 10 two PPCG inner steps in one pass, 11/12 four Chebyshev iterations in one pass (2D,
// FP64/FP32).
TEA_EXPORT void tea_kernel_timing_(const int* chunk, const int* kernel, const int* reps, double* ms_per_launch)
{
    *ms_per_launch = 0.0;
    Chunk* c = get_chunk(chunk);
    if (!c || *reps < 1) return;
    // Coefficient arrays for at least kTimingIters iterations, so that a pass of four
    // Chebyshev iterations reads stored coefficients even before any solve has run.
    constexpr int kTimingIters = 8;
    Fused* F = ensure_fused(c, kTimingIters);
    if (*kernel >= 7 && !ensure_fp32(c, F)) return;
    FusedArgs a = F->base;
    a.step = 1;
    a.timing = 1;
    // Steady-state operands: sweep A applies a pending p and u update, as it does in every
    // CG iteration after the first; the Chebyshev kernels see iterations that are neither
    // a convergence check nor past max_iters, so the four-iteration pass runs as a pass of
    // four (with max_iters below 4 it falls back to its two-iteration body).
    pull_state(c, F);
    const SolveState saved = *F->h_st;
    F->h_st->pending_p = 1;
    F->h_st->pending_u = 1;
    F->h_st->n = 1;
    F->h_st->cont = 1;
    F->h_st->est_itc = 1 << 30;
    F->h_st->max_iters = std::max(F->h_st->max_iters, kTimingIters);
    F->h_st->cheby_calc_steps = 1;
    F->h_st->n_inner = 1;
    F->h_st->inner_max = 1 << 30;
    push_state(c, F);
    cudaEvent_t e0, e1;
    TEA_CK(cudaEventCreate(&e0));
    TEA_CK(cudaEventCreate(&e1));
    auto launch = [&]() {
        switch (*kernel) {
        case 1: stencil<OpPPCGInner<false>>(F, a, c->stream); break;
        case 2: stencil<OpSweepA>(F, a, c->stream); break;
        case 3: stencil<OpCheby>(F, a, c->stream); break;
        case 5: k_cg_sweep_b<<<F->pair_blocks, 256, 0, c->stream>>>(a); break;
        case 7: stencil<OpSweepA32>(F, a, c->stream); break;
        case 8: k_cg32_sweep_b<<<F->quad_blocks, 256, 0, c->stream>>>(a); break;
#if TEA_DIM == 2
        case 9:
            if (F->pair32.blocks > 0) {
                FusedArgs ap = a;
                ap.seg_rows = F->pair32.rows;
                k_cheby2_ring2d<OpCheby32>
                    <<<F->pair32.blocks, RWARPS * 32, cheby2_smem_bytes<OpCheby32>(), c->stream>>>(ap);
            } else {
                stencil<OpCheby32>(F, a, c->stream);
            }
            break;
#else
        case 9: stencil<OpCheby32>(F, a, c->stream); break;
        case 6: stencil<OpCheby>(F, a, c->stream); break;
#endif
#if TEA_DIM == 2
        case 6:
            if (F->pair.blocks > 0) {
                FusedArgs ap = a;
                ap.seg_rows = F->pair.rows;
                k_cheby2_ring2d<OpCheby><<<F->pair.blocks, RWARPS * 32, cheby2_smem_bytes<OpCheby>(), c->stream>>>(ap);
            } else {
                stencil<OpCheby>(F, a, c->stream);
            }
            break;
#endif
#if TEA_DIM == 2
        case 11:
        case 12:
            if (F->quad.blocks > 0) {
                FusedArgs ap = a;
                if (*kernel == 11) {
                    launch_cheby4(F, a, saved.precond != 0, c->stream);
                } else {
                    ap.seg_rows = F->quad32.rows;
                    k_cheby4_ring2d<OpCheby32>
                        <<<F->quad32.blocks, RWARPS * 32, cheby4_smem_bytes<OpCheby32>(false), c->stream>>>(ap);
                }
            }
            break;
        case 10:
            if (F->ppcg2.blocks > 0) {
                FusedArgs ap = a;
                ap.seg_rows = F->ppcg2.rows;
                k_ppcg2_ring2d<PpcgF64><<<F->ppcg2.blocks, RWARPS * 32, ppcg2_2d_smem_bytes, c->stream>>>(ap);
            }
            break;
        case 13:
            if (F->ppcg2_32.blocks > 0) {
                FusedArgs ap = a;
                ap.seg_rows = F->ppcg2_32.rows;
                k_ppcg2_ring2d<PpcgF32><<<F->ppcg2_32.blocks, RWARPS * 32, ppcg2_2d_smem_bytes, c->stream>>>(ap);
            }
            break;
#else
        case 10:
            if (F->ppcg2.blocks > 0) launch_ppcg2_3d(F, a, saved.precond != 0, c->stream);
            break;
        case 13:
            if (F->ppcg2_32.blocks > 0) {
                FusedArgs ap = a;
                ap.seg_rows = F->ppcg2_32.rows;
                k_ppcg2_ring3d<PpcgF32, PPCG2_TY, PPCG2_RP_PLAIN, false><<<F->ppcg2_32.blocks, PPCG2_TY * 32,
                                                                          ppcg2_smem_bytes<float, PPCG2_TY,
                                                                                           PPCG2_RP_PLAIN, false>(),
                                                                          c->stream>>>(ap);
            }
            break;
#endif
        default: stencil<OpJacobi>(F, a, c->stream); break;
        }
    };
    launch();  // warm-up
    TEA_CK(cudaEventRecord(e0, c->stream));
    for (int k = 0; k < *reps; ++k) launch();
    TEA_CK(cudaEventRecord(e1, c->stream));
    TEA_CK(cudaEventSynchronize(e1));
    float ms = 0.0f;
    TEA_CK(cudaEventElapsedTime(&ms, e0, e1));
    *ms_per_launch = (double)ms / *reps;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *F->h_st = saved;
    push_state(c, F);
    sync(c);
}
