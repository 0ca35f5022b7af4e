/*
 * ORACLE -- test infrastructure only.  Never linked into, loaded by, or called from
 * the product path (libtea{2,3}d_b200.so, the driver).  Only tests/, the smoke check
 * and bench.py's CPU-baseline leg load it, to compare the CUDA library's results with.
 *
 * A plain-C, single-threaded restatement of the reference's extension kernels
 * (crtrott/TeaLeaf-Kokkos tealeaf_2d|3d/ext_*.hpp functors and the ext_* entry points
 * of ext_core.cpp / ext_chunk.cpp), exporting the same C ABI as the CUDA library so
 * that the same C++ driver runs on either.  Compiled twice: -DTEA_DIM=2 and -DTEA_DIM=3.
 *
 * Layout and arithmetic are the reference's: flat arrays of (nx+4)(ny+4)[(nz+4)]
 * doubles, x fastest (tealeaf_2d/ext_shared.hpp:43-45, tealeaf_3d/ext_shared.hpp:47-50),
 * every expression evaluated in the reference's order with FP contraction off.
 * Functors whose parallel_for visits every padded index but guards on a region are
 * restated as loops over that region in index order, which is the order a
 * single-thread Kokkos::OpenMP dispatch visits them.
 *
 * Reductions have two modes (oracle_set_sum_mode):
 *   0  TEA_SUM_SEQUENTIAL: acc = 0; acc += term in index order.  This is exactly
 *      Kokkos::OpenMP parallel_reduce with one thread
 *      (kokkos_src/core/src/OpenMP/Kokkos_OpenMP_Parallel.hpp:118-184), so the port is
 *      bit-identical to oracle/_ref run with OMP_NUM_THREADS=1.
 *   1  TEA_SUM_COMPENSATED: the terms are accumulated in double-double (Ogita-Rump-Oishi
 *      cascaded summation) and rounded once.  The result is the correctly rounded sum
 *      except when the exact sum lies within ~n*2^-106 (relative) of a rounding
 *      boundary, so it does not depend on the summation order.  The CUDA library sums
 *      this way, which makes the port and the GPU agree bit for bit.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifndef TEA_DIM
#error "compile with -DTEA_DIM=2 or -DTEA_DIM=3"
#endif

#define HALO_PAD 2
#define EXTERNAL_FACE -1
#define CONDUCTIVITY 1
#define RECIP_CONDUCTIVITY 2
#define MAX_CHUNKS 16

#define EXPORT __attribute__((visibility("default")))

typedef struct {
    int x, y, z;
} Dims;

typedef struct {
    Dims dims;
    long full;   /* padded length */
    long page;   /* dims.x*dims.y */
    int rank;
    double dx, dy, dz, theta;
    int preconditioner;
    double *density, *energy0, *energy, *u, *u0, *p, *r, *mi, *w, *z, *kx, *ky, *kz, *sd,
        *volume;
    double *vertexX, *vertexY, *vertexZ, *cellX, *cellY, *cellZ;
    double *alphas, *betas;
    int ncoefs;
} Chunk;

static Chunk* g_chunks[MAX_CHUNKS];
static int g_nchunks = 0;
static int g_sum_mode = 0;
static int g_status = 0;

EXPORT void oracle_set_sum_mode(int mode) { g_sum_mode = mode; }
EXPORT int oracle_get_sum_mode(void) { return g_sum_mode; }

EXPORT void ext_get_status_(int* status)
{
    *status = g_status;
    g_status = 0;
}
EXPORT const char* tea_last_error(void) { return ""; }

static void fatal(const char* msg, int value)
{
    /* The reference prints and exit(1)s: tealeaf_2d/ext_core.cpp:571-584. */
    fprintf(stderr, "\nError in tea_oracle: %s %d\n", msg, value);
    exit(1);
}

static Chunk* get_chunk(const int* chunk)
{
    if (*chunk < 1 || *chunk > g_nchunks || !g_chunks[*chunk - 1]) fatal("bad chunk", *chunk);
    return g_chunks[*chunk - 1];
}

/* ---------------------------------------------------------------- reductions */

typedef struct {
    double hi, lo;
} Acc;

static inline void acc_init(Acc* a)
{
    a->hi = 0.0;
    a->lo = 0.0;
}

static inline void acc_add(Acc* a, double x)
{
    if (g_sum_mode == 0) {
        a->hi += x;
        return;
    }
    /* TwoSum (Knuth): s + e == hi + x exactly. */
    double s = a->hi + x;
    double bp = s - a->hi;
    double e = (a->hi - (s - bp)) + (x - bp);
    a->hi = s;
    a->lo += e;
}

static inline double acc_value(const Acc* a) { return g_sum_mode == 0 ? a->hi : a->hi + a->lo; }

/* ---------------------------------------------------------------- indexing */

#if TEA_DIM == 2
#define IDX(c, kk, jj, ii) ((long)(kk) + (long)(jj) * (c)->dims.x)
#define ZLO(c) 0
#define ZHI(c) 1
#else
#define IDX(c, kk, jj, ii) ((long)(kk) + ((long)(jj) + (long)(ii) * (c)->dims.y) * (c)->dims.x)
#define ZLO(c) HALO_PAD
#define ZHI(c) ((c)->dims.z - HALO_PAD)
#endif

/* Inner domain (INDEX_IN_INNER_DOMAIN, tealeaf_2d/ext_shared.hpp:47-49). */
#define FOR_INNER(c)                                                  \
    for (int ii = ZLO(c); ii < ZHI(c); ++ii)                          \
        for (int jj = HALO_PAD; jj < (c)->dims.y - HALO_PAD; ++jj)    \
            for (int kk = HALO_PAD; kk < (c)->dims.x - HALO_PAD; ++kk)

/* The stencil SMVP(a) of tealeaf_2d/ext_shared.hpp:37-41 / tealeaf_3d/ext_shared.hpp:39-45
 * (Kx/Ky/Kz already carry rx/ry/rz). */
static inline double smvp(const Chunk* c, const double* a, long i)
{
    const double* kx = c->kx;
    const double* ky = c->ky;
    const long dx = c->dims.x;
#if TEA_DIM == 2
    return (1.0 + (kx[i + 1] + kx[i]) + (ky[i + dx] + ky[i])) * a[i]
        - (kx[i + 1] * a[i + 1] + kx[i] * a[i - 1])
        - (ky[i + dx] * a[i + dx] + ky[i] * a[i - dx]);
#else
    const double* kz = c->kz;
    const long pg = c->page;
    return (1.0 + (kx[i + 1] + kx[i]) + (ky[i + dx] + ky[i]) + (kz[i + pg] + kz[i])) * a[i]
        - (kx[i + 1] * a[i + 1] + kx[i] * a[i - 1])
        - (ky[i + dx] * a[i + dx] + ky[i] * a[i - dx])
        - (kz[i + pg] * a[i + pg] + kz[i] * a[i - pg]);
#endif
}

/* ---------------------------------------------------------------- chunk table */

static double* zalloc(long n)
{
    double* p = (double*)calloc((size_t)n, sizeof(double));
    if (!p) fatal("out of memory", 0);
    return p;
}

static Chunk* new_chunk(int x, int y, int z, int rank)
{
    /* TeaLeafChunk ctor, tealeaf_2d/ext_chunk.cpp:36-82, tealeaf_3d/ext_chunk.cpp:39-103:
     * every View is zero-initialised. */
    Chunk* c = (Chunk*)calloc(1, sizeof(Chunk));
    c->rank = rank;
    c->dims.x = x + 2 * HALO_PAD;
    c->dims.y = y + 2 * HALO_PAD;
    c->dims.z = TEA_DIM == 3 ? z + 2 * HALO_PAD : 1;
    c->page = (long)c->dims.x * c->dims.y;
    c->full = c->page * c->dims.z;
    double** fields[] = {&c->density, &c->energy0, &c->energy, &c->u,  &c->u0,
                         &c->p,       &c->r,       &c->mi,     &c->w,  &c->z,
                         &c->kx,      &c->ky,      &c->kz,     &c->sd, &c->volume};
    for (size_t f = 0; f < sizeof(fields) / sizeof(fields[0]); ++f) *fields[f] = zalloc(c->full);
    c->vertexX = zalloc(c->dims.x + 1);
    c->vertexY = zalloc(c->dims.y + 1);
    c->vertexZ = zalloc(c->dims.z + 1);
    c->cellX = zalloc(c->dims.x);
    c->cellY = zalloc(c->dims.y);
    c->cellZ = zalloc(c->dims.z);
    return c;
}

static void free_chunk(Chunk* c)
{
    double* fields[] = {c->density, c->energy0, c->energy, c->u,  c->u0, c->p,  c->r,
                        c->mi,      c->w,       c->z,      c->kx, c->ky, c->kz, c->sd,
                        c->volume,  c->vertexX, c->vertexY, c->vertexZ, c->cellX, c->cellY,
                        c->cellZ,   c->alphas,  c->betas};
    for (size_t f = 0; f < sizeof(fields) / sizeof(fields[0]); ++f) free(fields[f]);
    free(c);
}

#if TEA_DIM == 2
EXPORT void ext_init_(int* xMax, int* yMax, int* rank)
{
    if (g_nchunks >= MAX_CHUNKS) fatal("too many chunks", g_nchunks);
    g_chunks[g_nchunks++] = new_chunk(*xMax, *yMax, 1, *rank);
}
#else
EXPORT void ext_init_(int* xMax, int* yMax, int* zMax, int* rank)
{
    if (g_nchunks >= MAX_CHUNKS) fatal("too many chunks", g_nchunks);
    g_chunks[g_nchunks++] = new_chunk(*xMax, *yMax, *zMax, *rank);
}
#endif

EXPORT void ext_finalise_(void)
{
    /* tealeaf_2d/ext_chunk.cpp:29-33 deletes every chunk; the table is also emptied
     * here so that one process can run several problems. */
    for (int i = 0; i < g_nchunks; ++i) free_chunk(g_chunks[i]);
    g_nchunks = 0;
}

/* ---------------------------------------------------------------- set-up */

/* InitialiseChunkVertices, tealeaf_2d/ext_initialise_chunk.hpp:13-61 (3D :13-76), run
 * over n = max(dims) indices.  The functor writes vertexX(index) and, in the same
 * iteration, reads vertexX(index+1) for cellX(index); in index order vertexX(index+1)
 * still holds its value from before the call (zero on the first call).  The port
 * reproduces that single-thread outcome exactly.  vertexX(dims.x) is written only
 * when dims.x < n. */
static void init_axis(double* vertex, double* cell, int dimsN, int n, double lo, double d)
{
    for (int index = 0; index < n; ++index) {
        if (index < dimsN + 1) vertex[index] = lo + d * (index - HALO_PAD);
        if (index < dimsN) cell[index] = 0.5 * (vertex[index] + vertex[index + 1]);
    }
}

#if TEA_DIM == 2
EXPORT void ext_initialise_chunk_(const int* chunk, const double* xMin, const double* yMin,
                                  const double* dx, const double* dy)
{
    Chunk* c = get_chunk(chunk);
    c->dx = *dx;
    c->dy = *dy;
    int n = c->dims.x > c->dims.y ? c->dims.x : c->dims.y;
    /* The reference updates x and y in the same iteration; the axes are independent. */
    init_axis(c->vertexX, c->cellX, c->dims.x, n, *xMin, *dx);
    init_axis(c->vertexY, c->cellY, c->dims.y, n, *yMin, *dy);
    /* InitialiseChunkAreas, tealeaf_2d/ext_initialise_chunk.hpp:63-90 (areas unused). */
    for (long i = 0; i < c->full; ++i) c->volume[i] = *dx * *dy;
}
#else
EXPORT void ext_initialise_chunk_(const int* chunk, const double* xMin, const double* yMin,
                                  const double* zMin, const double* dx, const double* dy,
                                  const double* dz)
{
    Chunk* c = get_chunk(chunk);
    c->dx = *dx;
    c->dy = *dy;
    c->dz = *dz;
    int n = c->dims.x > c->dims.y ? c->dims.x : c->dims.y;
    n = n > c->dims.z ? n : c->dims.z;
    init_axis(c->vertexX, c->cellX, c->dims.x, n, *xMin, *dx);
    init_axis(c->vertexY, c->cellY, c->dims.y, n, *yMin, *dy);
    init_axis(c->vertexZ, c->cellZ, c->dims.z, n, *zMin, *dz);
    /* tealeaf_3d/ext_initialise_chunk.hpp:78-85: volume = dx*dy*dz. */
    for (long i = 0; i < c->full; ++i) c->volume[i] = *dx * *dy * *dz;
}
#endif

/* GenerateChunk, tealeaf_2d/ext_generate_chunk.hpp:13-101 (3D :13-109): every padded
 * cell starts in state 1; states 2..N are applied in order (last wins); u = e0*rho on
 * the one-cell halo domain. */
static void generate(Chunk* c, int nStates, const double* sDen, const double* sEn,
                     const double* sXMin, const double* sXMax, const double* sYMin,
                     const double* sYMax, const double* sZMin, const double* sZMax,
                     const double* sRad, const int* sGeo, int rect, int circ, int point)
{
    for (int ii = 0; ii < c->dims.z; ++ii)
        for (int jj = 0; jj < c->dims.y; ++jj)
            for (int kk = 0; kk < c->dims.x; ++kk) {
                long i = IDX(c, kk, jj, ii);
                c->energy0[i] = sEn[0];
                c->density[i] = sDen[0];
                for (int ss = 1; ss < nStates; ++ss) {
                    int apply = 0;
                    if (sGeo[ss] == rect) {
                        apply = c->vertexX[kk + 1] >= sXMin[ss] && c->vertexX[kk] < sXMax[ss]
                            && c->vertexY[jj + 1] >= sYMin[ss] && c->vertexY[jj] < sYMax[ss];
#if TEA_DIM == 3
                        apply = apply && c->vertexZ[ii + 1] >= sZMin[ss]
                            && c->vertexZ[ii] < sZMax[ss];
#endif
                    } else if (sGeo[ss] == circ) {
#if TEA_DIM == 2
                        double radius = sqrt((c->cellX[kk] - sXMin[ss]) * (c->cellX[kk] - sXMin[ss])
                                             + (c->cellY[jj] - sYMin[ss]) * (c->cellY[jj] - sYMin[ss]));
#else
                        double radius = sqrt((c->cellX[kk] - sXMin[ss]) * (c->cellX[kk] - sXMin[ss])
                                             + (c->cellY[jj] - sYMin[ss]) * (c->cellY[jj] - sYMin[ss])
                                             + (c->cellZ[ii] - sZMin[ss]) * (c->cellZ[ii] - sZMin[ss]));
#endif
                        apply = radius <= sRad[ss];
                    } else if (sGeo[ss] == point) {
                        apply = c->vertexX[kk] == sXMin[ss] && c->vertexY[jj] == sYMin[ss];
#if TEA_DIM == 3
                        apply = apply && c->vertexZ[ii] == sZMin[ss];
#endif
                    }
                    if (apply) {
                        c->energy0[i] = sEn[ss];
                        c->density[i] = sDen[ss];
                    }
                }
                int one = kk > 0 && kk < c->dims.x - 1 && jj > 0 && jj < c->dims.y - 1;
#if TEA_DIM == 3
                one = one && ii > 0 && ii < c->dims.z - 1;
#endif
                if (one) c->u[i] = c->energy0[i] * c->density[i];
            }
    (void)sZMin;
    (void)sZMax;
}

#if TEA_DIM == 2
EXPORT void ext_generate_chunk_(const int* chunk, const int* numStates,
                                const double* stateDensity, const double* stateEnergy,
                                const double* stateXMin, const double* stateXMax,
                                const double* stateYMin, const double* stateYMax,
                                const double* stateRadius, const int* stateGeometry,
                                const int* rectParam, const int* circParam, const int* pointParam)
{
    generate(get_chunk(chunk), *numStates, stateDensity, stateEnergy, stateXMin, stateXMax,
             stateYMin, stateYMax, NULL, NULL, stateRadius, stateGeometry, *rectParam,
             *circParam, *pointParam);
}
#else
EXPORT void ext_generate_chunk_(const int* chunk, const int* numStates,
                                const double* stateDensity, const double* stateEnergy,
                                const double* stateXMin, const double* stateXMax,
                                const double* stateYMin, const double* stateYMax,
                                const double* stateZMin, const double* stateZMax,
                                const double* stateRadius, const int* stateGeometry,
                                const int* rectParam, const int* circParam, const int* pointParam)
{
    generate(get_chunk(chunk), *numStates, stateDensity, stateEnergy, stateXMin, stateXMax,
             stateYMin, stateYMax, stateZMin, stateZMax, stateRadius, stateGeometry,
             *rectParam, *circParam, *pointParam);
}
#endif

/* FieldSummary, tealeaf_2d/ext_field_summary.hpp:13-67: ie uses energy0, temp uses u. */
EXPORT void ext_field_summary_kernel_(const int* chunk, double* vol, double* mass, double* ie,
                                      double* temp)
{
    Chunk* c = get_chunk(chunk);
    Acc a_vol, a_mass, a_ie, a_temp;
    acc_init(&a_vol);
    acc_init(&a_mass);
    acc_init(&a_ie);
    acc_init(&a_temp);
    FOR_INNER(c)
    {
        long i = IDX(c, kk, jj, ii);
        double cellVol = c->volume[i];
        double cellMass = cellVol * c->density[i];
        acc_add(&a_vol, cellVol);
        acc_add(&a_mass, cellMass);
        acc_add(&a_ie, cellMass * c->energy0[i]);
        acc_add(&a_temp, cellMass * c->u[i]);
    }
    *vol = acc_value(&a_vol);
    *mass = acc_value(&a_mass);
    *ie = acc_value(&a_ie);
    *temp = acc_value(&a_temp);
}

/* ---------------------------------------------------------------- halo / packing */

static double* halo_field(Chunk* c, int id)
{
    /* FIELD_* ids, tealeaf_2d/ext_shared.hpp:19-25. */
    switch (id) {
    case 1: return c->density;
    case 2: return c->energy0;
    case 3: return c->energy;
    case 4: return c->u;
    case 5: return c->p;
    case 6: return c->sd;
    default: fatal("Incorrect field provided:", id);
    }
    return NULL;
}

/* UpdateHalo, tealeaf_2d/ext_update_halo.hpp:12-76 (3D :12-136): reflective copy
 * halo[HALO_PAD-1-f] = interior[HALO_PAD+f] for f < depth.  In 2D the left/right faces
 * span every row (halo rows included) and run before top/bottom, which span every
 * column; in 3D only the inner part of each face is written. */
static void update_face(Chunk* c, double* b, int face, int depth)
{
    const int X = c->dims.x, Y = c->dims.y;
#if TEA_DIM == 2
    switch (face) {
    case 1: /* CHUNK_LEFT */
        for (int jj = 0; jj < Y; ++jj)
            for (int f = 0; f < depth; ++f) b[(HALO_PAD - 1 - f) + (long)jj * X] = b[(HALO_PAD + f) + (long)jj * X];
        break;
    case 2: /* CHUNK_RIGHT */
        for (int jj = 0; jj < Y; ++jj)
            for (int f = 0; f < depth; ++f)
                b[(X - HALO_PAD + f) + (long)jj * X] = b[(X - HALO_PAD - 1 - f) + (long)jj * X];
        break;
    case 4: /* CHUNK_TOP */
        for (int f = 0; f < depth; ++f)
            for (int kk = 0; kk < X; ++kk)
                b[kk + (long)(Y - HALO_PAD + f) * X] = b[kk + (long)(Y - HALO_PAD - 1 - f) * X];
        break;
    case 3: /* CHUNK_BOTTOM */
        for (int f = 0; f < depth; ++f)
            for (int kk = 0; kk < X; ++kk)
                b[kk + (long)(HALO_PAD - 1 - f) * X] = b[kk + (long)(HALO_PAD + f) * X];
        break;
    }
#else
    const int Z = c->dims.z;
    switch (face) {
    case 1: /* CHUNK_LEFT */
        for (int ii = HALO_PAD; ii < Z - HALO_PAD; ++ii)
            for (int jj = HALO_PAD; jj < Y - HALO_PAD; ++jj)
                for (int f = 0; f < depth; ++f)
                    b[IDX(c, HALO_PAD - 1 - f, jj, ii)] = b[IDX(c, HALO_PAD + f, jj, ii)];
        break;
    case 2: /* CHUNK_RIGHT */
        for (int ii = HALO_PAD; ii < Z - HALO_PAD; ++ii)
            for (int jj = HALO_PAD; jj < Y - HALO_PAD; ++jj)
                for (int f = 0; f < depth; ++f)
                    b[IDX(c, X - HALO_PAD + f, jj, ii)] = b[IDX(c, X - HALO_PAD - 1 - f, jj, ii)];
        break;
    case 4: /* CHUNK_TOP */
        for (int ii = HALO_PAD; ii < Z - HALO_PAD; ++ii)
            for (int f = 0; f < depth; ++f)
                for (int kk = HALO_PAD; kk < X - HALO_PAD; ++kk)
                    b[IDX(c, kk, Y - HALO_PAD + f, ii)] = b[IDX(c, kk, Y - HALO_PAD - 1 - f, ii)];
        break;
    case 3: /* CHUNK_BOTTOM */
        for (int ii = HALO_PAD; ii < Z - HALO_PAD; ++ii)
            for (int f = 0; f < depth; ++f)
                for (int kk = HALO_PAD; kk < X - HALO_PAD; ++kk)
                    b[IDX(c, kk, HALO_PAD - 1 - f, ii)] = b[IDX(c, kk, HALO_PAD + f, ii)];
        break;
    case 6: /* CHUNK_FRONT */
        for (int f = 0; f < depth; ++f)
            for (int jj = HALO_PAD; jj < Y - HALO_PAD; ++jj)
                for (int kk = HALO_PAD; kk < X - HALO_PAD; ++kk)
                    b[IDX(c, kk, jj, Z - HALO_PAD + f)] = b[IDX(c, kk, jj, Z - HALO_PAD - 1 - f)];
        break;
    case 5: /* CHUNK_BACK */
        for (int f = 0; f < depth; ++f)
            for (int jj = HALO_PAD; jj < Y - HALO_PAD; ++jj)
                for (int kk = HALO_PAD; kk < X - HALO_PAD; ++kk)
                    b[IDX(c, kk, jj, HALO_PAD - 1 - f)] = b[IDX(c, kk, jj, HALO_PAD + f)];
        break;
    }
#endif
}

EXPORT void ext_update_halo_kernel_(const int* chunk, const int* chunkNeighbours,
                                    const int* fields, const int* depth)
{
    Chunk* c = get_chunk(chunk);
    /* Field order of the dispatch, tealeaf_2d/ext_core.cpp:330-335 (order is
     * immaterial: the arrays are independent).  Face order per field: left, right,
     * top, bottom [, front, back] (:324-327, tealeaf_3d/ext_core.cpp:353-358). */
    static const int order[6] = {1, 5, 2, 3, 4, 6};
#if TEA_DIM == 2
    static const int faces[4] = {1, 2, 4, 3};
    const int nfaces = 4;
#else
    static const int faces[6] = {1, 2, 4, 3, 6, 5};
    const int nfaces = 6;
#endif
    for (int o = 0; o < 6; ++o) {
        int f = order[o];
        if (!fields[f - 1]) continue;
        double* b = halo_field(c, f);
        for (int q = 0; q < nfaces; ++q)
            if (chunkNeighbours[faces[q] - 1] == EXTERNAL_FACE) update_face(c, b, faces[q], *depth);
    }
}

/* Packers, tealeaf_2d/ext_pack_kernel.hpp:8-97 and tealeaf_3d/ext_pack_kernel.hpp.
 * The field index of buffer element `index` is restated from each packer's offset
 * expression; 3D front/back follow tealeaf_3d/ext_pack_kernel.hpp:137-190. */
static long pack_index(const Chunk* c, int face, int depth, int pack, long index, int exact)
{
    const long X = c->dims.x, Y = c->dims.y;
#if TEA_DIM == 2
    if (face == 1 || face == 2) {
        long lines = index / depth;
        long off;
        if (face == 1) off = pack ? HALO_PAD + lines * (X - depth) : HALO_PAD - depth + lines * (X - depth);
        else off = pack ? X - HALO_PAD - depth + lines * (X - depth) : X - HALO_PAD + lines * (X - depth);
        return off + index;
    } else {
        long width = X - 2 * HALO_PAD;
        long lines = index / width;
        long off;
        if (face == 4) off = pack ? X * (Y - HALO_PAD - depth) + lines * 2 * HALO_PAD
                                  : X * (Y - HALO_PAD) + lines * 2 * HALO_PAD;
        else off = pack ? X * HALO_PAD + lines * 2 * HALO_PAD : X * (HALO_PAD - depth) + lines * 2 * HALO_PAD;
        return off + index + (exact ? HALO_PAD : 0);
    }
#else
    (void)exact;
    const long Z = c->dims.z;
    const long HP2 = 2 * HALO_PAD;
    const long page = X * Y;
    if (face == 1 || face == 2) {
        long height = Y - HP2;
        long lines = index / depth;
        long base = page * HALO_PAD + X * HALO_PAD + lines * (X - depth) + (lines / height) * X * HP2;
        long xoff;
        if (face == 1) xoff = pack ? HALO_PAD : HALO_PAD - depth;
        else xoff = pack ? X - HALO_PAD - depth : X - HALO_PAD;
        return base + xoff + index;
    } else if (face == 3 || face == 4) {
        long width = X - HP2;
        long lines = index / width;
        long yoff;
        if (face == 4) yoff = pack ? X * (Y - HALO_PAD - depth) : X * (Y - HALO_PAD);
        else yoff = pack ? X * HALO_PAD : X * (HALO_PAD - depth);
        return page * HALO_PAD + yoff + HALO_PAD + lines * HP2 + X * (Y - depth) * (lines / depth) + index;
    } else {
        long height = Y - HP2;
        long lines = index / (X - HP2);
        long zoff;
        if (face == 6) zoff = pack ? page * (Z - HALO_PAD - depth) : page * (Z - HALO_PAD);
        else zoff = pack ? page * HALO_PAD : page * (HALO_PAD - depth);
        return zoff + X * HALO_PAD + HALO_PAD + lines * HP2 + (lines / height) * X * HP2 + index;
    }
#endif
}

static void pack_message(Chunk* c, const int* fields, const int* offsets, int depth, int face,
                         double* buffer, int pack, int exact)
{
    long len;
#if TEA_DIM == 2
    if (face == 1 || face == 2) len = (long)(c->dims.y - 2 * HALO_PAD) * depth;
    else if (face == 3 || face == 4) len = (long)(c->dims.x - 2 * HALO_PAD) * depth;
    else { fatal("Incorrect face provided:", face); return; }
#else
    long nx = c->dims.x - 2 * HALO_PAD, ny = c->dims.y - 2 * HALO_PAD, nz = c->dims.z - 2 * HALO_PAD;
    if (face == 1 || face == 2) len = ny * nz * depth;
    else if (face == 3 || face == 4) len = nx * nz * depth;
    else if (face == 5 || face == 6) len = nx * ny * depth;
    else { fatal("Incorrect face provided:", face); return; }
#endif
    for (int f = 0; f < 6; ++f) {
        if (!fields[f]) continue;
        double* b = halo_field(c, f + 1);
        double* ext = buffer + offsets[f];
        for (long index = 0; index < len; ++index) {
            long fi = pack_index(c, face, depth, pack, index, exact);
            if (pack) ext[index] = b[fi];
            else b[fi] = ext[index];
        }
    }
}

#if TEA_DIM == 2
EXPORT void ext_pack_message_(const int* chunk, const int* fields, const int* offsets,
                              const int* depth, const int* face, double* buffer,
                              const void* pack)
{
    pack_message(get_chunk(chunk), fields, offsets, *depth, *face, buffer,
                 *(const unsigned char*)pack != 0, 0);
}
#else
EXPORT void ext_pack_message_(const int* chunk, const int* fields, const int* offsets,
                              const int* depth, const int* face, const int* fieldType,
                              double* buffer, const void* pack)
{
    (void)fieldType;
    pack_message(get_chunk(chunk), fields, offsets, *depth, *face, buffer,
                 *(const unsigned char*)pack != 0, 0);
}
#endif

/* The exchange packer of the slab driver: ext_pack_message_ with the 2D bottom/top faces
 * on the inner columns (the reference's 2D packer starts at column 0,
 * tealeaf_2d/ext_pack_kernel.hpp:17-44); 3D faces are identical to it. */
EXPORT void tea_pack_face_(const int* chunk, const int* fields, const int* offsets, const int* depth,
                           const int* face, double* buffer, const void* pack)
{
    pack_message(get_chunk(chunk), fields, offsets, *depth, *face, buffer, *(const unsigned char*)pack != 0, 1);
}


/* ---------------------------------------------------------------- shared methods */

/* SetField, tealeaf_2d/ext_set_field.hpp:13-29: whole padded array. */
EXPORT void ext_set_field_kernel_(const int* chunk)
{
    Chunk* c = get_chunk(chunk);
    for (long i = 0; i < c->full; ++i) c->energy[i] = c->energy0[i];
}

/* CopyU, tealeaf_2d/ext_solver_methods.hpp:12-35. */
EXPORT void ext_solver_copy_u_(const int* chunk)
{
    Chunk* c = get_chunk(chunk);
    FOR_INNER(c) { long i = IDX(c, kk, jj, ii); c->u0[i] = c->u[i]; }
}

/* CalculateResidual, tealeaf_2d/ext_solver_methods.hpp:38-66. */
EXPORT void ext_calculate_residual_(const int* chunk)
{
    Chunk* c = get_chunk(chunk);
    FOR_INNER(c)
    {
        long i = IDX(c, kk, jj, ii);
        const double s = smvp(c, c->u, i);
        c->r[i] = c->u0[i] - s;
    }
}

/* Calculate2Norm, tealeaf_2d/ext_solver_methods.hpp:70-92; buffer chosen at
 * tealeaf_2d/ext_core.cpp:289. */
EXPORT void ext_calculate_2norm_(const int* chunk, double* norm, const void* normArray)
{
    Chunk* c = get_chunk(chunk);
    const double* b = *(const unsigned char*)normArray ? c->r : c->u0;
    Acc a;
    acc_init(&a);
    FOR_INNER(c) { long i = IDX(c, kk, jj, ii); acc_add(&a, b[i] * b[i]); }
    *norm = acc_value(&a);
}

/* Finalise, tealeaf_2d/ext_solver_methods.hpp:96-121. */
EXPORT void ext_solver_finalise_(const int* chunk)
{
    Chunk* c = get_chunk(chunk);
    FOR_INNER(c) { long i = IDX(c, kk, jj, ii); c->energy[i] = c->u[i] / c->density[i]; }
}

/* ---------------------------------------------------------------- Jacobi */

/* JacobiInit, tealeaf_2d/ext_jacobi_kernel.hpp:12-62 (3D :12-66). */
EXPORT void ext_jacobi_kernel_init_(const int* chunk, const int* coefficient, const double* dt)
{
    Chunk* c = get_chunk(chunk);
    if (*coefficient < CONDUCTIVITY && *coefficient < RECIP_CONDUCTIVITY)
        fatal("Coefficient is not valid.", *coefficient);
    const double rx = *dt / (c->dx * c->dx);
    const double ry = *dt / (c->dy * c->dy);
#if TEA_DIM == 3
    const double rz = *dt / (c->dz * c->dz);
#endif
    const int cond = *coefficient == CONDUCTIVITY;
    const long dx = c->dims.x;
    for (int ii = 0; ii < c->dims.z; ++ii)
        for (int jj = 0; jj < c->dims.y; ++jj)
            for (int kk = 0; kk < c->dims.x; ++kk) {
                long i = IDX(c, kk, jj, ii);
                int one = jj > 0 && jj < c->dims.y - 1 && kk > 0 && kk < c->dims.x - 1;
                int skew = jj >= HALO_PAD && jj < c->dims.y - 1 && kk >= HALO_PAD && kk < c->dims.x - 1;
#if TEA_DIM == 3
                one = one && ii > 0 && ii < c->dims.z - 1;
                skew = skew && ii >= HALO_PAD && ii < c->dims.z - 1;
#endif
                if (one) {
                    c->u0[i] = c->energy[i] * c->density[i];
                    c->u[i] = c->u0[i];
                }
                if (skew) {
                    double centre = cond ? c->density[i] : 1.0 / c->density[i];
                    double left = cond ? c->density[i - 1] : 1.0 / c->density[i - 1];
                    double down = cond ? c->density[i - dx] : 1.0 / c->density[i - dx];
                    c->kx[i] = rx * (left + centre) / (2.0 * left * centre);
                    c->ky[i] = ry * (down + centre) / (2.0 * down * centre);
#if TEA_DIM == 3
                    double back = cond ? c->density[i - c->page] : 1.0 / c->density[i - c->page];
                    c->kz[i] = rz * (back + centre) / (2.0 * back * centre);
#endif
                }
            }
}

/* JacobiCopyU + JacobiSolve, tealeaf_2d/ext_jacobi_kernel.hpp:66-117 (3D :70-126). */
EXPORT void ext_jacobi_kernel_solve_(const int* chunk, double* error)
{
    Chunk* c = get_chunk(chunk);
    memcpy(c->r, c->u, sizeof(double) * (size_t)c->full);
    const double *kx = c->kx, *ky = c->ky, *r = c->r;
    const long dx = c->dims.x;
#if TEA_DIM == 3
    const double* kz = c->kz;
    const long pg = c->page;
#endif
    Acc a;
    acc_init(&a);
    FOR_INNER(c)
    {
        long i = IDX(c, kk, jj, ii);
#if TEA_DIM == 2
        c->u[i] = (c->u0[i] + (kx[i + 1] * r[i + 1] + kx[i] * r[i - 1])
                   + (ky[i + dx] * r[i + dx] + ky[i] * r[i - dx]))
            / (1.0 + (kx[i] + kx[i + 1]) + (ky[i] + ky[i + dx]));
#else
        c->u[i] = (c->u0[i] + (kx[i + 1] * r[i + 1] + kx[i] * r[i - 1])
                   + (ky[i + dx] * r[i + dx] + ky[i] * r[i - dx])
                   + (kz[i + pg] * r[i + pg] + kz[i] * r[i - pg]))
            / (1.0 + (kx[i] + kx[i + 1]) + (ky[i] + ky[i + dx]) + (kz[i] + kz[i + pg]));
#endif
        acc_add(&a, fabs(c->u[i] - r[i]));
    }
    *error = acc_value(&a);
}

/* ---------------------------------------------------------------- CG */

EXPORT void ext_cg_solver_init_(const int* chunk, const int* coefficient, const int* preconditioner,
                                double* dt, double* rro)
{
    Chunk* c = get_chunk(chunk);
    if (*coefficient < CONDUCTIVITY && *coefficient < RECIP_CONDUCTIVITY)
        fatal("Coefficient is not valid.", *coefficient);
    c->preconditioner = *preconditioner;
    /* CGInitU, tealeaf_2d/ext_cg_kernel.hpp:13-34: whole padded array. */
    for (long i = 0; i < c->full; ++i) {
        c->p[i] = 0.0;
        c->r[i] = 0.0;
        c->u[i] = c->energy[i] * c->density[i];
    }
    const double rx = *dt / (c->dx * c->dx);
    const double ry = *dt / (c->dy * c->dy);
#if TEA_DIM == 3
    const double rz = *dt / (c->dz * c->dz);
#endif
    const long dx = c->dims.x;
    /* CGInitW, tealeaf_2d/ext_cg_kernel.hpp:37-61: one-cell halo domain. */
    for (int ii = (TEA_DIM == 3 ? 1 : 0); ii < (TEA_DIM == 3 ? c->dims.z - 1 : 1); ++ii)
        for (int jj = 1; jj < c->dims.y - 1; ++jj)
            for (int kk = 1; kk < c->dims.x - 1; ++kk) {
                long i = IDX(c, kk, jj, ii);
                c->w[i] = (*coefficient == CONDUCTIVITY) ? c->density[i] : 1.0 / c->density[i];
            }
    /* CGInitK, tealeaf_2d/ext_cg_kernel.hpp:64-91 (3D :60-91): skew domain. */
    for (int ii = (TEA_DIM == 3 ? HALO_PAD : 0); ii < (TEA_DIM == 3 ? c->dims.z - 1 : 1); ++ii)
        for (int jj = HALO_PAD; jj < c->dims.y - 1; ++jj)
            for (int kk = HALO_PAD; kk < c->dims.x - 1; ++kk) {
                long i = IDX(c, kk, jj, ii);
                const double* w = c->w;
                c->kx[i] = rx * (w[i - 1] + w[i]) / (2.0 * w[i - 1] * w[i]);
                c->ky[i] = ry * (w[i - dx] + w[i]) / (2.0 * w[i - dx] * w[i]);
#if TEA_DIM == 3
                c->kz[i] = rz * (w[i - c->page] + w[i]) / (2.0 * w[i - c->page] * w[i]);
#endif
            }
    /* CGCalcRRO, tealeaf_2d/ext_cg_kernel.hpp:94-145 (3D :94-149). */
    Acc a;
    acc_init(&a);
    FOR_INNER(c)
    {
        long i = IDX(c, kk, jj, ii);
        const double s = smvp(c, c->u, i);
        c->w[i] = s;
        c->r[i] = c->u[i] - c->w[i];
        if (c->preconditioner) {
#if TEA_DIM == 2
            c->mi[i] = (1.0 + (c->kx[i + 1] + c->kx[i]) + (c->ky[i + dx] + c->ky[i]));
#else
            c->mi[i] = (1.0 + (c->kx[i + 1] + c->kx[i]) + (c->ky[i + dx] + c->ky[i])
                        + (c->kz[i + c->page] + c->kz[i]));
#endif
            c->mi[i] = 1.0 / c->mi[i];
            c->z[i] = c->mi[i] * c->r[i];
            c->p[i] = c->z[i];
        } else {
            c->p[i] = c->r[i];
        }
        acc_add(&a, c->r[i] * c->p[i]);
    }
    *rro = acc_value(&a);
}

/* CGCalcW, tealeaf_2d/ext_cg_kernel.hpp:148-197 (non-team path :177-189). */
EXPORT void ext_cg_calc_w_(const int* chunk, double* pw)
{
    Chunk* c = get_chunk(chunk);
    Acc a;
    acc_init(&a);
    FOR_INNER(c)
    {
        long i = IDX(c, kk, jj, ii);
        const double s = smvp(c, c->p, i);
        c->w[i] = s;
        acc_add(&a, c->w[i] * c->p[i]);
    }
    *pw = acc_value(&a);
}

/* CGCalcUr, tealeaf_2d/ext_cg_kernel.hpp:200-275 (non-team path :244-264). */
EXPORT void ext_cg_calc_ur_(const int* chunk, const double* alpha, double* rrn)
{
    Chunk* c = get_chunk(chunk);
    const double al = *alpha;
    Acc a;
    acc_init(&a);
    FOR_INNER(c)
    {
        long i = IDX(c, kk, jj, ii);
        c->u[i] += al * c->p[i];
        c->r[i] -= al * c->w[i];
        if (c->preconditioner) {
            c->z[i] = c->mi[i] * c->r[i];
            acc_add(&a, c->r[i] * c->z[i]);
        } else {
            acc_add(&a, c->r[i] * c->r[i]);
        }
    }
    *rrn = acc_value(&a);
}

/* CGCalcP, tealeaf_2d/ext_cg_kernel.hpp:278-319 (non-team path :301-310). */
EXPORT void ext_cg_calc_p_(const int* chunk, const double* beta)
{
    Chunk* c = get_chunk(chunk);
    const double b = *beta;
    FOR_INNER(c)
    {
        long i = IDX(c, kk, jj, ii);
        c->p[i] = b * c->p[i] + (c->preconditioner ? c->z[i] : c->r[i]);
    }
}

/* ---------------------------------------------------------------- Chebyshev */

static void store_coefs(Chunk* c, const double* alphas, const double* betas, int n)
{
    free(c->alphas);
    free(c->betas);
    c->alphas = zalloc(n > 0 ? n : 1);
    c->betas = zalloc(n > 0 ? n : 1);
    memcpy(c->alphas, alphas, sizeof(double) * (size_t)n);
    memcpy(c->betas, betas, sizeof(double) * (size_t)n);
    c->ncoefs = n;
}

static void cheby_calc_u(Chunk* c)
{
    /* ChebyCalcU, tealeaf_2d/ext_cheby_kernel.hpp:50-72. */
    FOR_INNER(c) { long i = IDX(c, kk, jj, ii); c->u[i] += c->p[i]; }
}

/* ext_cheby_solver_init_, tealeaf_2d/ext_core.cpp:468-497: ChebyInit
 * (tealeaf_2d/ext_cheby_kernel.hpp:11-47) then ChebyCalcU. */
EXPORT void ext_cheby_solver_init_(const int* chunk, double* alphas, double* betas,
                                   const double* theta, const int* preconditioner,
                                   const int* maxChebyIters)
{
    Chunk* c = get_chunk(chunk);
    c->preconditioner = *preconditioner;
    store_coefs(c, alphas, betas, *maxChebyIters);
    const double th = *theta;
    FOR_INNER(c)
    {
        long i = IDX(c, kk, jj, ii);
        const double s = smvp(c, c->u, i);
        c->w[i] = s;
        c->r[i] = c->u0[i] - c->w[i];
        c->p[i] = (c->preconditioner ? c->mi[i] * c->r[i] : c->r[i]) / th;
    }
    cheby_calc_u(c);
}

/* ext_cheby_solver_iterate_, tealeaf_2d/ext_core.cpp:501-515: ChebyIterate
 * (tealeaf_2d/ext_cheby_kernel.hpp:75-115) with step = chebyCalcStep-1, then ChebyCalcU. */
EXPORT void ext_cheby_solver_iterate_(const int* chunk, const int* chebyCalcStep)
{
    Chunk* c = get_chunk(chunk);
    const int step = *chebyCalcStep - 1;
    if (step < 0 || step >= c->ncoefs) fatal("Chebyshev step out of range:", step);
    const double al = c->alphas[step], be = c->betas[step];
    FOR_INNER(c)
    {
        long i = IDX(c, kk, jj, ii);
        const double s = smvp(c, c->u, i);
        c->w[i] = s;
        c->r[i] = c->u0[i] - c->w[i];
        c->p[i] = al * c->p[i] + be * (c->preconditioner ? c->mi[i] * c->r[i] : c->r[i]);
    }
    cheby_calc_u(c);
}

/* ---------------------------------------------------------------- PPCG */

/* ext_ppcg_init_, tealeaf_2d/ext_core.cpp:519-539. */
EXPORT void ext_ppcg_init_(const int* chunk, double* alphas, double* betas, const double* theta,
                           const int* maxChebyIters)
{
    Chunk* c = get_chunk(chunk);
    c->theta = *theta;
    store_coefs(c, alphas, betas, *maxChebyIters);
}

/* PPCGInitSd, tealeaf_2d/ext_ppcg_kernel.hpp:8-34. */
EXPORT void ext_ppcg_init_sd_(const int* chunk)
{
    Chunk* c = get_chunk(chunk);
    FOR_INNER(c)
    {
        long i = IDX(c, kk, jj, ii);
        c->sd[i] = (c->preconditioner ? c->mi[i] * c->r[i] : c->r[i]) / c->theta;
    }
}

/* ext_ppcg_inner_, tealeaf_2d/ext_core.cpp:554-567: PPCGCalcU
 * (tealeaf_2d/ext_ppcg_kernel.hpp:37-65) then PPCGCalcSd (:68-100) with step-1. */
EXPORT void ext_ppcg_inner_(const int* chunk, int* currentStep)
{
    Chunk* c = get_chunk(chunk);
    const int step = *currentStep - 1;
    if (step < 0 || step >= c->ncoefs) fatal("PPCG step out of range:", step);
    FOR_INNER(c)
    {
        long i = IDX(c, kk, jj, ii);
        const double s = smvp(c, c->sd, i);
        c->r[i] -= s;
        c->u[i] += c->sd[i];
    }
    const double al = c->alphas[step], be = c->betas[step];
    FOR_INNER(c)
    {
        long i = IDX(c, kk, jj, ii);
        c->sd[i] = al * c->sd[i] + be * (c->preconditioner ? c->mi[i] * c->r[i] : c->r[i]);
    }
}

/* ---------------------------------------------------------------- inspection */

static double* any_field(Chunk* c, int id)
{
    switch (id) {
    case 1: return c->density;
    case 2: return c->energy0;
    case 3: return c->energy;
    case 4: return c->u;
    case 5: return c->p;
    case 6: return c->sd;
    case 7: return c->u0;
    case 8: return c->r;
    case 9: return c->w;
    case 10: return c->z;
    case 11: return c->mi;
    case 12: return c->kx;
    case 13: return c->ky;
    case 14: return TEA_DIM == 3 ? c->kz : NULL;
    case 15: return c->volume;
    default: return NULL;
    }
}

EXPORT int tea_chunk_dims_(const int* chunk, int* dims)
{
    if (*chunk < 1 || *chunk > g_nchunks) return 1;
    Chunk* c = g_chunks[*chunk - 1];
    dims[0] = c->dims.x;
    dims[1] = c->dims.y;
    dims[2] = c->dims.z;
    return 0;
}

EXPORT int tea_read_field_(const int* chunk, const int* field, double* out)
{
    if (*chunk < 1 || *chunk > g_nchunks) return 1;
    Chunk* c = g_chunks[*chunk - 1];
    double* f = any_field(c, *field);
    if (!f) return 1;
    memcpy(out, f, sizeof(double) * (size_t)c->full);
    return 0;
}

EXPORT int tea_write_field_(const int* chunk, const int* field, const double* in)
{
    if (*chunk < 1 || *chunk > g_nchunks) return 1;
    Chunk* c = g_chunks[*chunk - 1];
    double* f = any_field(c, *field);
    if (!f) return 1;
    memcpy(f, in, sizeof(double) * (size_t)c->full);
    return 0;
}
