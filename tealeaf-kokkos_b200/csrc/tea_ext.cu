// The drop-in C ABI of the TeaLeaf B200 library (include/tea_ext_2d.h, tea_ext_3d.h,
// tea_b200.h).  Compiled once per dimension: -DTEA_DIM=2 -> libtea2d_b200.so,
// -DTEA_DIM=3 -> libtea3d_b200.so.  An entry point that hands data to the host (a
// reduction, a field summary, a packed face, a field read) returns once its kernels have
// finished; one that only updates fields returns once they are queued on the chunk's
// stream, as the reference's Kokkos parallel_for dispatches do (tealeaf_2d/ext_core.cpp:21-24).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "tea_chunk.cuh"
#include "tea_kernels.cuh"

#define TEA_EXPORT extern "C" __attribute__((visibility("default")))

namespace tea {

std::vector<Chunk*>& chunks()
{
    static std::vector<Chunk*> v;
    return v;
}

Chunk* get_chunk(const int* chunk)
{
    auto& v = chunks();
    if (!chunk || *chunk < 1 || (size_t)*chunk > v.size() || !v[*chunk - 1]) {
        set_status(1, "invalid chunk id %d", chunk ? *chunk : -1);
        return nullptr;
    }
    return v[*chunk - 1];
}

static bool verbose()
{
    static int v = -1;
    if (v < 0) v = std::getenv("TEA_B200_VERBOSE") ? 1 : 0;
    return v == 1;
}

double* field_ptr(Chunk* c, int id)
{
    if (id < 1 || id >= F_COUNT) return nullptr;
    if (id == F_KZ && DIM != 3) return nullptr;
    return c->alloc[id] ? c->alloc[id] + kLeadPad : nullptr;
}

// Synchronise the chunk's stream and report launch/runtime errors.
void sync(Chunk* c)
{
    TEA_CK(cudaGetLastError());
    TEA_CK(cudaStreamSynchronize(c->stream));
}

// End of an entry point that only updates fields: launch errors are reported now, faults
// inside its kernels at the next synchronisation (the next reduction, field read or
// ext_get_status_).
static void issued(Chunk*)
{
    TEA_CK(cudaGetLastError());
}

Chunk* create_chunk(int nx, int ny, int nz, int rank)
{
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        set_status(6, "no CUDA device available (%s): the TeaLeaf B200 library has no CPU path",
                   cudaGetErrorString(e));
        return nullptr;
    }
    if (nx < 1 || ny < 1 || nz < 1) {
        set_status(2, "invalid chunk size %d x %d x %d", nx, ny, nz);
        return nullptr;
    }
    Chunk* c = new Chunk();
    c->rank = rank;
    TEA_CK(cudaGetDevice(&c->device));
    Geom& g = c->g;
    g.nx = nx;
    g.ny = ny;
    g.nz = DIM == 3 ? nz : 1;
    g.X = nx + 2 * HALO_PAD;
    g.Y = ny + 2 * HALO_PAD;
    g.Z = DIM == 3 ? nz + 2 * HALO_PAD : 1;
    g.pitch = ((long)g.X + kPitchAlign - 1) / kPitchAlign * kPitchAlign;
    g.page = g.pitch * g.Y;
    c->inner = make_box(HALO_PAD, g.X - HALO_PAD, HALO_PAD, g.Y - HALO_PAD, DIM == 3 ? HALO_PAD : 0,
                        DIM == 3 ? g.Z - HALO_PAD : 1);
    c->full = make_box(0, g.X, 0, g.Y, 0, g.Z);
    c->one = make_box(1, g.X - 1, 1, g.Y - 1, DIM == 3 ? 1 : 0, DIM == 3 ? g.Z - 1 : 1);
    c->skew = make_box(HALO_PAD, g.X - 1, HALO_PAD, g.Y - 1, DIM == 3 ? HALO_PAD : 0, DIM == 3 ? g.Z - 1 : 1);
    g.tiles_x = c->inner.tx;
    g.tiles_y = c->inner.ty;
    g.tiles_inner = c->inner.ntiles;
    g.ftiles_x = c->full.tx;
    g.ftiles_y = c->full.ty;
    g.tiles_full = c->full.ntiles;
    // Every array is zero-initialised, as Kokkos Views are.  Trailing slack of one pitch
    // keeps vector loads of the last row inside the allocation.
    c->field_elems = (size_t)kLeadPad + (size_t)g.page * g.Z + (size_t)g.pitch;
    for (int id = 1; id < F_COUNT; ++id) {
        if (id == F_KZ && DIM != 3) continue;
        TEA_CK(cudaMalloc(&c->alloc[id], c->field_elems * sizeof(double)));
        if (c->alloc[id]) TEA_CK(cudaMemset(c->alloc[id], 0, c->field_elems * sizeof(double)));
    }
    Fields& f = c->f;
    f.density = field_ptr(c, F_DENSITY);
    f.energy0 = field_ptr(c, F_ENERGY0);
    f.energy = field_ptr(c, F_ENERGY1);
    f.u = field_ptr(c, F_U);
    f.p = field_ptr(c, F_P);
    f.sd = field_ptr(c, F_SD);
    f.u0 = field_ptr(c, F_U0);
    f.r = field_ptr(c, F_R);
    f.w = field_ptr(c, F_W);
    f.z = field_ptr(c, F_Z);
    f.mi = field_ptr(c, F_MI);
    f.kx = field_ptr(c, F_KX);
    f.ky = field_ptr(c, F_KY);
    f.kz = DIM == 3 ? field_ptr(c, F_KZ) : nullptr;
    f.volume = field_ptr(c, F_VOLUME);
    c->vx.assign(g.X + 1, 0.0);
    c->vy.assign(g.Y + 1, 0.0);
    c->vz.assign(g.Z + 1, 0.0);
    c->cx.assign(g.X, 0.0);
    c->cy.assign(g.Y, 0.0);
    c->cz.assign(g.Z, 0.0);
    TEA_CK(cudaMalloc(&c->d_vx, sizeof(double) * (g.X + 1)));
    TEA_CK(cudaMalloc(&c->d_vy, sizeof(double) * (g.Y + 1)));
    TEA_CK(cudaMalloc(&c->d_vz, sizeof(double) * (g.Z + 1)));
    TEA_CK(cudaMalloc(&c->d_cx, sizeof(double) * g.X));
    TEA_CK(cudaMalloc(&c->d_cy, sizeof(double) * g.Y));
    TEA_CK(cudaMalloc(&c->d_cz, sizeof(double) * g.Z));
    TEA_CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    int sms = 148;
    TEA_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
    c->grid_blocks = sms * 8;
    c->red.max_blocks = c->grid_blocks;
    TEA_CK(cudaMalloc(&c->red.partials, sizeof(DD) * MAX_RED * c->red.max_blocks));
    TEA_CK(cudaMalloc(&c->red.counter, sizeof(unsigned int)));
    TEA_CK(cudaMemset(c->red.counter, 0, sizeof(unsigned int)));
    TEA_CK(cudaHostAlloc(&c->h_out, 8 * sizeof(double), cudaHostAllocMapped));
    TEA_CK(cudaHostGetDevicePointer(&c->d_out, c->h_out, 0));
    TEA_CK(cudaDeviceSynchronize());
    if (rank == 0 && verbose()) {
        if (DIM == 2) std::printf("Problem Size: %dx%d\n", nx, ny);
        else std::printf("Problem Size: %dx%dx%d\n", nx, ny, nz);
    }
    return c;
}

void destroy_fused(Chunk* c);  // tea_fused.cu

void destroy_chunk(Chunk* c)
{
    if (!c) return;
    destroy_fused(c);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (int id = 1; id < F_COUNT; ++id)
        if (c->alloc[id]) cudaFree(c->alloc[id]);
    double* small[] = {c->d_vx, c->d_vy, c->d_vz, c->d_cx, c->d_cy, c->d_cz};
    for (double* p : small)
        if (p) cudaFree(p);
    if (c->red.partials) cudaFree(c->red.partials);
    if (c->red.counter) cudaFree(c->red.counter);
    if (c->h_out) cudaFreeHost(c->h_out);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

// Result of a reduction kernel written through the mapped pointer.
double result(Chunk* c, int k)
{
    sync(c);
    c->d2h_bytes += sizeof(double);
    return ((volatile double*)c->h_out)[k];
}

void store_coefs(Chunk* c, const double* alphas, const double* betas, int n)
{
    if (n < 1) n = 1;
    c->h_alphas.assign(alphas, alphas + n);
    c->h_betas.assign(betas, betas + n);
    c->h2d_bytes += 2 * sizeof(double) * (long long)n;
}

// InitialiseChunkVertices, tealeaf_2d/ext_initialise_chunk.hpp:13-61: computed on the
// host (a few thousand values).  The functor writes vertex(index) and reads
// vertex(index+1) in the same iteration, so cell(index) sees the value vertex(index+1)
// held before the call; a single-threaded dispatch of the reference produces exactly
// this, and it is reproduced here deterministically.  vertex(n) stays untouched when
// the axis is the longest one.
void init_axis(std::vector<double>& vertex, std::vector<double>& cell, int dimsN, int n, double lo, double d)
{
    for (int index = 0; index < n; ++index) {
        if (index < dimsN + 1) vertex[index] = lo + d * (index - HALO_PAD);
        if (index < dimsN) cell[index] = 0.5 * (vertex[index] + vertex[index + 1]);
    }
}

void upload_coords(Chunk* c)
{
    const Geom& g = c->g;
    TEA_CK(copy_on(c->stream, c->d_vx, c->vx.data(), sizeof(double) * (g.X + 1), cudaMemcpyHostToDevice));
    TEA_CK(copy_on(c->stream, c->d_vy, c->vy.data(), sizeof(double) * (g.Y + 1), cudaMemcpyHostToDevice));
    TEA_CK(copy_on(c->stream, c->d_vz, c->vz.data(), sizeof(double) * (g.Z + 1), cudaMemcpyHostToDevice));
    TEA_CK(copy_on(c->stream, c->d_cx, c->cx.data(), sizeof(double) * g.X, cudaMemcpyHostToDevice));
    TEA_CK(copy_on(c->stream, c->d_cy, c->cy.data(), sizeof(double) * g.Y, cudaMemcpyHostToDevice));
    TEA_CK(copy_on(c->stream, c->d_cz, c->cz.data(), sizeof(double) * g.Z, cudaMemcpyHostToDevice));
}

void initialise_chunk(Chunk* c, double xmin, double ymin, double zmin, double dx, double dy, double dz)
{
    c->dx = dx;
    c->dy = dy;
    c->dz = dz;
    const Geom& g = c->g;
    int n = std::max(g.X, g.Y);
    if (DIM == 3) n = std::max(n, g.Z);
    init_axis(c->vx, c->cx, g.X, n, xmin, dx);
    init_axis(c->vy, c->cy, g.Y, n, ymin, dy);
    if (DIM == 3) init_axis(c->vz, c->cz, g.Z, n, zmin, dz);
    upload_coords(c);
    const double vol = DIM == 3 ? dx * dy * dz : dx * dy;
    k_init_volume<<<launch_blocks(c, c->full.ntiles), dim3(TILE_X, TILE_Y), 0, c->stream>>>(c->g, c->full,
                                                                                          c->f.volume, vol);
    sync(c);
}

void generate_chunk(Chunk* c, int n, const double* den, const double* en, const double* x0, const double* x1,
                    const double* y0, const double* y1, const double* z0, const double* z1, const double* rad,
                    const int* geo, int rect, int circ, int point)
{
    if (n < 1) {
        set_status(2, "ext_generate_chunk_: no states");
        return;
    }
    // Pack the state tables into one device buffer.
    std::vector<double> h(9 * (size_t)n, 0.0);
    for (int s = 0; s < n; ++s) {
        h[0 * n + s] = den[s];
        h[1 * n + s] = en[s];
        h[2 * n + s] = x0[s];
        h[3 * n + s] = x1[s];
        h[4 * n + s] = y0[s];
        h[5 * n + s] = y1[s];
        h[6 * n + s] = z0 ? z0[s] : 0.0;
        h[7 * n + s] = z1 ? z1[s] : 0.0;
        h[8 * n + s] = rad[s];
    }
    double* d = nullptr;
    int* dg = nullptr;
    TEA_CK(cudaMalloc(&d, sizeof(double) * h.size()));
    TEA_CK(cudaMalloc(&dg, sizeof(int) * n));
    TEA_CK(copy_on(c->stream, d, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice));
    TEA_CK(copy_on(c->stream, dg, geo, sizeof(int) * n, cudaMemcpyHostToDevice));
    c->h2d_bytes += (long long)(sizeof(double) * h.size() + sizeof(int) * n);
    StateTable st;
    st.n = n;
    st.rect = rect;
    st.circ = circ;
    st.point = point;
    st.density = d;
    st.energy = d + n;
    st.xmin = d + 2 * n;
    st.xmax = d + 3 * n;
    st.ymin = d + 4 * n;
    st.ymax = d + 5 * n;
    st.zmin = d + 6 * n;
    st.zmax = d + 7 * n;
    st.radius = d + 8 * n;
    st.geometry = dg;
    k_generate<<<launch_blocks(c, c->full.ntiles), dim3(TILE_X, TILE_Y), 0, c->stream>>>(
        c->g, c->full, c->f, st, c->d_vx, c->d_vy, c->d_vz, c->d_cx, c->d_cy, c->d_cz);
    sync(c);
    TEA_CK(cudaFree(d));
    TEA_CK(cudaFree(dg));
}

double* halo_field(Chunk* c, int id)
{
    switch (id) {
    case 1: return c->f.density;
    case 2: return c->f.energy0;
    case 3: return c->f.energy;
    case 4: return c->f.u;
    case 5: return c->f.p;
    case 6: return c->f.sd;
    default: return nullptr;
    }
}

void update_halo(Chunk* c, const int* neighbours, const int* fields, int depth)
{
    const Geom& g = c->g;
    if (depth < 1 || depth > HALO_PAD) {
        set_status(2, "ext_update_halo_kernel_: depth %d outside 1..%d", depth, HALO_PAD);
        return;
    }
    // Two phases in 2D (left/right span the halo rows that top/bottom then copy); one in 3D.
    const int nphase = DIM == 2 ? 2 : 1;
    for (int phase = 0; phase < nphase; ++phase) {
        HaloJob job;
        job.nseg = 0;
        job.depth = depth;
        long maxcount = 0;
        for (int fid = 1; fid <= 6; ++fid) {
            if (!fields[fid - 1]) continue;
            double* b = halo_field(c, fid);
            const int nf = DIM == 2 ? 4 : 6;
            for (int face = 1; face <= nf; ++face) {
                if (neighbours[face - 1] != -1) continue;
                long count;
                if (DIM == 2) {
                    const bool lr = face <= 2;
                    if ((phase == 0) != lr) continue;
                    count = lr ? (long)g.Y * depth : (long)g.X * depth;
                } else {
                    if (face <= 2) count = (long)g.ny * g.nz * depth;
                    else if (face <= 4) count = (long)g.nx * g.nz * depth;
                    else count = (long)g.nx * g.ny * depth;
                }
                job.seg[job.nseg].field = b;
                job.seg[job.nseg].face = face;
                job.seg[job.nseg].count = count;
                ++job.nseg;
                maxcount = std::max(maxcount, count);
            }
        }
        if (job.nseg == 0) continue;
        const int threads = 256;
        long bx = (maxcount + threads - 1) / threads;
        bx = std::min<long>(bx, 4096);
        k_update_halo<<<dim3((unsigned)std::max<long>(bx, 1), job.nseg), threads, 0, c->stream>>>(c->g, job);
    }
    issued(c);
}

}  // namespace tea

using namespace tea;

// ===================================================================== chunk table

#if TEA_DIM == 2
TEA_EXPORT void ext_init_(int* xMax, int* yMax, int* rank)
{
    Chunk* c = create_chunk(*xMax, *yMax, 1, *rank);
    if (c) chunks().push_back(c);
}
#else
TEA_EXPORT void ext_init_(int* xMax, int* yMax, int* zMax, int* rank)
{
    Chunk* c = create_chunk(*xMax, *yMax, *zMax, *rank);
    if (c) chunks().push_back(c);
}
#endif

TEA_EXPORT void ext_finalise_(void)
{
    // The reference deletes every chunk (tealeaf_2d/ext_chunk.cpp:29-33); the table is
    // emptied as well so that a process can set up another problem afterwards.
    for (Chunk* c : chunks()) destroy_chunk(c);
    chunks().clear();
}

// ===================================================================== set-up

#if TEA_DIM == 2
TEA_EXPORT void ext_initialise_chunk_(const int* chunk, const double* xMin, const double* yMin,
                                      const double* dx, const double* dy)
{
    Chunk* c = get_chunk(chunk);
    if (c) initialise_chunk(c, *xMin, *yMin, 0.0, *dx, *dy, 0.0);
}

TEA_EXPORT void ext_generate_chunk_(const int* chunk, const int* numStates, const double* stateDensity,
                                    const double* stateEnergy, const double* stateXMin, const double* stateXMax,
                                    const double* stateYMin, const double* stateYMax, const double* stateRadius,
                                    const int* stateGeometry, const int* rectParam, const int* circParam,
                                    const int* pointParam)
{
    Chunk* c = get_chunk(chunk);
    if (c)
        generate_chunk(c, *numStates, stateDensity, stateEnergy, stateXMin, stateXMax, stateYMin, stateYMax,
                       nullptr, nullptr, stateRadius, stateGeometry, *rectParam, *circParam, *pointParam);
}
#else
TEA_EXPORT void ext_initialise_chunk_(const int* chunk, const double* xMin, const double* yMin,
                                      const double* zMin, const double* dx, const double* dy, const double* dz)
{
    Chunk* c = get_chunk(chunk);
    if (c) initialise_chunk(c, *xMin, *yMin, *zMin, *dx, *dy, *dz);
}

TEA_EXPORT void ext_generate_chunk_(const int* chunk, const int* numStates, const double* stateDensity,
                                    const double* stateEnergy, const double* stateXMin, const double* stateXMax,
                                    const double* stateYMin, const double* stateYMax, const double* stateZMin,
                                    const double* stateZMax, const double* stateRadius, const int* stateGeometry,
                                    const int* rectParam, const int* circParam, const int* pointParam)
{
    Chunk* c = get_chunk(chunk);
    if (c)
        generate_chunk(c, *numStates, stateDensity, stateEnergy, stateXMin, stateXMax, stateYMin, stateYMax,
                       stateZMin, stateZMax, stateRadius, stateGeometry, *rectParam, *circParam, *pointParam);
}
#endif

TEA_EXPORT void ext_field_summary_kernel_(const int* chunk, double* vol, double* mass, double* ie, double* temp)
{
    Chunk* c = get_chunk(chunk);
    if (!c) return;
    k_field_summary<<<launch_blocks(c, c->inner.ntiles), dim3(TILE_X, TILE_Y), 0, c->stream>>>(
        c->g, c->inner, c->f, c->red, c->d_out);
    sync(c);
    c->d2h_bytes += 4 * sizeof(double);
    volatile double* h = c->h_out;
    *vol = h[0];
    *mass = h[1];
    *ie = h[2];
    *temp = h[3];
}

// ===================================================================== halo / pack

static void pack_message(const int* chunk, const int* fields, const int* offsets, const int* depth,
                         const int* face, double* buffer, const void* pack, bool exact = false)
{
    Chunk* c = get_chunk(chunk);
    if (!c) return;
    const bool do_pack = *(const unsigned char*)pack != 0;
    const Geom& g = c->g;
    long len;
    if (*face == 1 || *face == 2) len = (long)g.ny * (DIM == 3 ? g.nz : 1) * *depth;
    else if (*face == 3 || *face == 4) len = (long)g.nx * (DIM == 3 ? g.nz : 1) * *depth;
    else if (DIM == 3 && (*face == 5 || *face == 6)) len = (long)g.nx * g.ny * *depth;
    else {
        set_status(2, "ext_pack_message_: Incorrect face provided: %d", *face);
        return;
    }
    double* dbuf = nullptr;
    TEA_CK(cudaMalloc(&dbuf, sizeof(double) * std::max<long>(len, 1)));
    for (int fid = 1; fid <= 6; ++fid) {
        if (!fields[fid - 1]) continue;
        double* ext = buffer + offsets[fid - 1];
        if (!do_pack) {
            TEA_CK(copy_on(c->stream, dbuf, ext, sizeof(double) * len, cudaMemcpyHostToDevice));
            c->h2d_bytes += (long long)sizeof(double) * len;
        }
        const int blocks = (int)std::min<long>((len + 255) / 256, 4096);
        k_pack<<<std::max(blocks, 1), 256, 0, c->stream>>>(c->g, halo_field(c, fid), dbuf, len, *face, *depth,
                                                           do_pack ? 1 : 0, exact ? 1 : 0);
        sync(c);
        if (do_pack) {
            TEA_CK(copy_on(c->stream, ext, dbuf, sizeof(double) * len, cudaMemcpyDeviceToHost));
            c->d2h_bytes += (long long)sizeof(double) * len;
        }
    }
    TEA_CK(cudaFree(dbuf));
}

#if TEA_DIM == 2
TEA_EXPORT void ext_pack_message_(const int* chunk, const int* fields, const int* offsets, const int* depth,
                                  const int* face, double* buffer, const void* pack)
{
    pack_message(chunk, fields, offsets, depth, face, buffer, pack);
}
#else
TEA_EXPORT void ext_pack_message_(const int* chunk, const int* fields, const int* offsets, const int* depth,
                                  const int* face, const int* fieldType, double* buffer, const void* pack)
{
    (void)fieldType;
    pack_message(chunk, fields, offsets, depth, face, buffer, pack);
}
#endif

// Face packing for an exchange between ranks: ext_pack_message_ with the 2D bottom/top faces
// on the inner columns (see pack_flat_index); 3D faces are identical to it.
TEA_EXPORT void tea_pack_face_(const int* chunk, const int* fields, const int* offsets, const int* depth,
                               const int* face, double* buffer, const void* pack)
{
    pack_message(chunk, fields, offsets, depth, face, buffer, pack, true);
}

TEA_EXPORT void ext_update_halo_kernel_(const int* chunk, const int* chunkNeighbours, const int* fields,
                                        const int* depth)
{
    Chunk* c = get_chunk(chunk);
    if (c) update_halo(c, chunkNeighbours, fields, *depth);
}

// ===================================================================== shared methods

#define LAUNCH(kernel, box, ...)                                                                   \
    kernel<<<launch_blocks(c, (box).ntiles), dim3(TILE_X, TILE_Y), 0, c->stream>>>(__VA_ARGS__)

// Segment-walk kernels (walk_cell_pairs): one warp per 64-cell row segment at most,
// 256-thread blocks, at most one wave of resident blocks (no partial second wave) and no
// more blocks than the reduction scratch holds partials for.
static int pair_blocks(const Chunk* c)
{
    static int wave = 0;  // blocks of one wave of the heaviest segment-walk kernel
    if (wave == 0) {
        int sms = 148, occ = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
        int n = 8;
        for (const void* k : {(const void*)k_cg_calc_w, (const void*)k_cheby_iterate, (const void*)k_ppcg_calc_u,
                              (const void*)k_jacobi_solve, (const void*)k_cg_calc_ur})
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, BLOCK, 0) == cudaSuccess && occ > 0)
                n = std::min(n, occ);
        wave = sms * n;
    }
    const long nseg = (long)((c->g.nx + 63) / 64) * c->g.ny * c->g.nz;
    return (int)std::max<long>(1, std::min<long>(std::min<long>((nseg + 7) / 8, wave), c->red.max_blocks));
}
#define LAUNCH_PAIRS(kernel, ...) kernel<<<pair_blocks(c), BLOCK, 0, c->stream>>>(__VA_ARGS__)

TEA_EXPORT void ext_set_field_kernel_(const int* chunk)
{
    Chunk* c = get_chunk(chunk);
    if (!c) return;
    LAUNCH(k_set_field, c->full, c->g, c->full, c->f);
    issued(c);
}

TEA_EXPORT void ext_solver_copy_u_(const int* chunk)
{
    Chunk* c = get_chunk(chunk);
    if (!c) return;
    LAUNCH_PAIRS(k_copy_u, c->g, c->f);
    issued(c);
}

TEA_EXPORT void ext_calculate_residual_(const int* chunk)
{
    Chunk* c = get_chunk(chunk);
    if (!c) return;
    LAUNCH_PAIRS(k_residual, c->g, c->f);
    issued(c);
}

TEA_EXPORT void ext_calculate_2norm_(const int* chunk, double* norm, const void* normArray)
{
    Chunk* c = get_chunk(chunk);
    if (!c) return;
    const double* b = *(const unsigned char*)normArray ? c->f.r : c->f.u0;
    LAUNCH_PAIRS(k_2norm, c->g, b, c->red, c->d_out);
    *norm = result(c, 0);
}

TEA_EXPORT void ext_solver_finalise_(const int* chunk)
{
    Chunk* c = get_chunk(chunk);
    if (!c) return;
    LAUNCH_PAIRS(k_finalise, c->g, c->f);
    issued(c);
}

// ===================================================================== Jacobi

static bool coefficient_ok(int coefficient)
{
    // The reference's test (tealeaf_2d/ext_core.cpp:347) is `< 1 && < 2`, i.e. only
    // values below 1 abort; anything else is treated as RECIP_CONDUCTIVITY unless 1.
    if (coefficient < 1 && coefficient < 2) {
        std::fprintf(stderr, "\nError: Coefficient %d is not valid.\n", coefficient);
        std::exit(1);
    }
    return true;
}

TEA_EXPORT void ext_jacobi_kernel_init_(const int* chunk, const int* coefficient, const double* dt)
{
    Chunk* c = get_chunk(chunk);
    if (!c || !coefficient_ok(*coefficient)) return;
    const double rx = *dt / (c->dx * c->dx);
    const double ry = *dt / (c->dy * c->dy);
    const double rz = DIM == 3 ? *dt / (c->dz * c->dz) : 0.0;
    LAUNCH(k_jacobi_init, c->full, c->g, c->full, c->f, *coefficient == 1 ? 1 : 0, rx, ry, rz);
    issued(c);
}

TEA_EXPORT void ext_jacobi_kernel_solve_(const int* chunk, double* error)
{
    Chunk* c = get_chunk(chunk);
    if (!c) return;
    k_jacobi_copy<<<pair_blocks(c), BLOCK, 0, c->stream>>>(c->g, c->f);
    LAUNCH_PAIRS(k_jacobi_solve, c->g, c->f, c->red, c->d_out);
    *error = result(c, 0);
}

// ===================================================================== CG

TEA_EXPORT void ext_cg_solver_init_(const int* chunk, const int* coefficient, const int* preconditioner, double* dt,
                                    double* rro)
{
    Chunk* c = get_chunk(chunk);
    if (!c || !coefficient_ok(*coefficient)) return;
    c->preconditioner = *preconditioner != 0;
    if (c->rank == 0 && verbose()) std::printf("Setting preconditioner to %d\n", *preconditioner);
    const double rx = *dt / (c->dx * c->dx);
    const double ry = *dt / (c->dy * c->dy);
    const double rz = DIM == 3 ? *dt / (c->dz * c->dz) : 0.0;
    LAUNCH(k_cg_init_uw, c->full, c->g, c->full, c->f, *coefficient == 1 ? 1 : 0);
    LAUNCH(k_cg_init_k, c->skew, c->g, c->skew, c->f, rx, ry, rz);
    LAUNCH(k_cg_calc_rro, c->inner, c->g, c->inner, c->f, c->preconditioner, c->red, c->d_out);
    *rro = result(c, 0);
}

TEA_EXPORT void ext_cg_calc_w_(const int* chunk, double* pw)
{
    Chunk* c = get_chunk(chunk);
    if (!c) return;
    LAUNCH_PAIRS(k_cg_calc_w, c->g, c->f, c->red, c->d_out);
    *pw = result(c, 0);
}

TEA_EXPORT void ext_cg_calc_ur_(const int* chunk, const double* alpha, double* rrn)
{
    Chunk* c = get_chunk(chunk);
    if (!c) return;
    LAUNCH_PAIRS(k_cg_calc_ur, c->g, c->f, *alpha, c->preconditioner, c->red, c->d_out);
    *rrn = result(c, 0);
}

TEA_EXPORT void ext_cg_calc_p_(const int* chunk, const double* beta)
{
    Chunk* c = get_chunk(chunk);
    if (!c) return;
    LAUNCH_PAIRS(k_cg_calc_p, c->g, c->f, *beta, c->preconditioner);
    issued(c);
}

// ===================================================================== Chebyshev

TEA_EXPORT void ext_cheby_solver_init_(const int* chunk, double* alphas, double* betas, const double* theta,
                                       const int* preconditioner, const int* maxChebyIters)
{
    Chunk* c = get_chunk(chunk);
    if (!c) return;
    c->preconditioner = *preconditioner != 0;
    store_coefs(c, alphas, betas, *maxChebyIters);
    LAUNCH(k_cheby_init, c->inner, c->g, c->inner, c->f, *theta, c->preconditioner);
    LAUNCH_PAIRS(k_cheby_calc_u, c->g, c->f);
    issued(c);
}

TEA_EXPORT void ext_cheby_solver_iterate_(const int* chunk, const int* chebyCalcStep)
{
    Chunk* c = get_chunk(chunk);
    if (!c) return;
    const int step = *chebyCalcStep - 1;
    if (step < 0 || step >= (int)c->h_alphas.size()) {
        set_status(2, "ext_cheby_solver_iterate_: step %d outside the %zu stored coefficients", step + 1,
                   c->h_alphas.size());
        return;
    }
    LAUNCH_PAIRS(k_cheby_iterate, c->g, c->f, c->h_alphas[step], c->h_betas[step],
           c->preconditioner);
    LAUNCH_PAIRS(k_cheby_calc_u, c->g, c->f);
    issued(c);
}

// ===================================================================== PPCG

TEA_EXPORT void ext_ppcg_init_(const int* chunk, double* alphas, double* betas, const double* theta,
                               const int* maxChebyIters)
{
    Chunk* c = get_chunk(chunk);
    if (!c) return;
    c->theta = *theta;
    store_coefs(c, alphas, betas, *maxChebyIters);
}

TEA_EXPORT void ext_ppcg_init_sd_(const int* chunk)
{
    Chunk* c = get_chunk(chunk);
    if (!c) return;
    LAUNCH_PAIRS(k_ppcg_init_sd, c->g, c->f, c->theta, c->preconditioner);
    issued(c);
}

TEA_EXPORT void ext_ppcg_inner_(const int* chunk, int* currentStep)
{
    Chunk* c = get_chunk(chunk);
    if (!c) return;
    const int step = *currentStep - 1;
    if (step < 0 || step >= (int)c->h_alphas.size()) {
        set_status(2, "ext_ppcg_inner_: step %d outside the %zu stored coefficients", step + 1, c->h_alphas.size());
        return;
    }
    LAUNCH_PAIRS(k_ppcg_calc_u, c->g, c->f);
    LAUNCH_PAIRS(k_ppcg_calc_sd, c->g, c->f, c->h_alphas[step], c->h_betas[step], c->preconditioner);
    issued(c);
}

// ===================================================================== inspection / status

TEA_EXPORT int tea_chunk_dims_(const int* chunk, int* dims)
{
    auto& v = chunks();
    if (!chunk || *chunk < 1 || (size_t)*chunk > v.size()) return 1;
    Chunk* c = v[*chunk - 1];
    dims[0] = c->g.X;
    dims[1] = c->g.Y;
    dims[2] = c->g.Z;
    return 0;
}

static int copy_field(const int* chunk, const int* field, double* host, bool to_host)
{
    auto& v = chunks();
    if (!chunk || *chunk < 1 || (size_t)*chunk > v.size()) return 1;
    Chunk* c = v[*chunk - 1];
    double* d = field_ptr(c, *field);
    if (!d) return 1;
    const Geom& g = c->g;
    // Rows of X doubles; the device rows are `pitch` apart, the host rows X apart.
    cudaError_t e;
    if (to_host)
        e = cudaMemcpy2DAsync(host, sizeof(double) * g.X, d, sizeof(double) * g.pitch, sizeof(double) * g.X,
                              (size_t)g.Y * g.Z, cudaMemcpyDeviceToHost, c->stream);
    else
        e = cudaMemcpy2DAsync(d, sizeof(double) * g.pitch, host, sizeof(double) * g.X, sizeof(double) * g.X,
                              (size_t)g.Y * g.Z, cudaMemcpyHostToDevice, c->stream);
    TEA_CK(e);
    sync(c);
    return e == cudaSuccess ? 0 : 1;
}

TEA_EXPORT int tea_read_field_(const int* chunk, const int* field, double* out)
{
    return copy_field(chunk, field, out, true);
}

TEA_EXPORT int tea_write_field_(const int* chunk, const int* field, const double* in)
{
    return copy_field(chunk, field, const_cast<double*>(in), false);
}

TEA_EXPORT void ext_get_status_(int* status)
{
    // Faults of kernels still queued by field-updating entry points are reported first.
    for (Chunk* c : chunks())
        if (c) sync(c);
    StatusStore& s = status_store();
    *status = s.status;
    s.status = 0;
}

TEA_EXPORT const char* tea_last_error(void) { return status_store().message.c_str(); }

// The chunk's CUDA stream (cudaStream_t), for callers that order their own work or
// record events after the library's.
TEA_EXPORT int tea_chunk_stream_(const int* chunk, void** stream)
{
    auto& v = chunks();
    if (!chunk || *chunk < 1 || (size_t)*chunk > v.size()) return 1;
    *stream = (void*)v[*chunk - 1]->stream;
    return 0;
}

// Host<->device bytes the library has moved for this chunk so far (state tables,
// coefficients, scalars, results, solve-state records); field arrays stay on the device.
TEA_EXPORT int tea_transfer_bytes_(const int* chunk, long long* h2d, long long* d2h)
{
    auto& v = chunks();
    if (!chunk || *chunk < 1 || (size_t)*chunk > v.size()) return 1;
    *h2d = v[*chunk - 1]->h2d_bytes;
    *d2h = v[*chunk - 1]->d2h_bytes;
    return 0;
}
