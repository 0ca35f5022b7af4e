// Test-infrastructure shim, linked only into oracle/_ref/libtea_ref{2,3}d.so.
//
// Gives the parity tests read/write access to the field arrays held by the
// reference's own chunk table (the global `Chunks` vector of
// tealeaf_2d/ext_chunk.cpp:15 / tealeaf_3d/ext_chunk.cpp:17) through the same
// inspection entry points that the CUDA library and the C port export
// (include/tea_b200.h: tea_chunk_dims_, tea_read_field_, tea_write_field_).
// The reference runs on Kokkos::OpenMP, so its Views live in host memory and
// are copied with memcpy.  Field ids follow include/tea_b200.h.
#include "ext_chunk.hpp"

#include <cstring>

namespace {

typedef Kokkos::View<double*, DEVICE> FieldView;

bool pick(TeaLeafChunk<DEVICE>* c, int field, FieldView& out)
{
    switch (field) {
    case 1: out = c->density; return true;
    case 2: out = c->energy0; return true;
    case 3: out = c->energy; return true;
    case 4: out = c->u; return true;
    case 5: out = c->p; return true;
    case 6: out = c->sd; return true;
    case 7: out = c->u0; return true;
    case 8: out = c->r; return true;
    case 9: out = c->w; return true;
    case 10: out = c->z; return true;
    case 11: out = c->mi; return true;
    case 12: out = c->kx; return true;
    case 13: out = c->ky; return true;
#if TEA_DIM == 3
    case 14: out = c->kz; return true;
#endif
    case 15: out = c->volume; return true;
    default: return false;
    }
}

TeaLeafChunk<DEVICE>* chunk_at(const int* chunk)
{
    if (!chunk || *chunk < 1 || (size_t)*chunk > Chunks.size()) return 0;
    return Chunks[*chunk - 1];
}

}  // namespace

extern "C" int tea_chunk_dims_(const int* chunk, int* dims)
{
    TeaLeafChunk<DEVICE>* c = chunk_at(chunk);
    if (!c) return 1;
    dims[0] = c->dims.x;
    dims[1] = c->dims.y;
#if TEA_DIM == 3
    dims[2] = c->dims.z;
#else
    dims[2] = 1;
#endif
    return 0;
}

extern "C" int tea_read_field_(const int* chunk, const int* field, double* out)
{
    TeaLeafChunk<DEVICE>* c = chunk_at(chunk);
    FieldView v;
    if (!c || !pick(c, *field, v)) return 1;
    std::memcpy(out, v.ptr_on_device(), sizeof(double) * c->fullDomain);
    return 0;
}

extern "C" int tea_write_field_(const int* chunk, const int* field, const double* in)
{
    TeaLeafChunk<DEVICE>* c = chunk_at(chunk);
    FieldView v;
    if (!c || !pick(c, *field, v)) return 1;
    std::memcpy(v.ptr_on_device(), in, sizeof(double) * c->fullDomain);
    return 0;
}

// ext_initialise_chunk_ with the cell centres a one-thread dispatch computes.
//
// InitialiseChunkVertices (tealeaf_2d/ext_initialise_chunk.hpp:13-61, tealeaf_3d: the
// same with z) writes vertex(index) and reads vertex(index + 1) in one parallel_for, so a
// cell centre depends on whether the thread owning index + 1 has run yet.  On one thread
// it never has: cell(i) = 0.5 * (vertex(i) + the value vertex(i + 1) held before the
// call).  On several OpenMP threads the cells at the ends of the threads' index ranges get
// the written value instead, and circles/spheres are painted differently along those
// columns, rows and planes.  This build renames the reference's entry point (objcopy in
// oracle/Makefile) and runs it through this wrapper, which recomputes the cell centres as
// the one-thread run does, so that fixtures recorded on several threads describe the same
// problem as one-thread runs (and as the oracle and the CUDA library, which follow the
// one-thread result).
#include <vector>

namespace {

std::vector<double> snapshot(const FieldView& v)
{
    std::vector<double> out(v.dimension_0());
    if (!out.empty()) std::memcpy(out.data(), v.ptr_on_device(), sizeof(double) * out.size());
    return out;
}

void one_thread_centres(const FieldView& vertex, const FieldView& cell, const std::vector<double>& old, int n)
{
    for (int i = 0; i < n; ++i) cell(i) = 0.5 * (vertex(i) + old[i + 1]);
}

}  // namespace

#if TEA_DIM == 2
extern "C" void ref_initialise_chunk_orig_(const int* chunk, const double* xMin, const double* yMin,
                                           const double* dx, const double* dy);

extern "C" void ext_initialise_chunk_(const int* chunk, const double* xMin, const double* yMin, const double* dx,
                                      const double* dy)
{
    TeaLeafChunk<DEVICE>* c = chunk_at(chunk);
    const std::vector<double> vx = snapshot(c->vertexX), vy = snapshot(c->vertexY);
    ref_initialise_chunk_orig_(chunk, xMin, yMin, dx, dy);
    one_thread_centres(c->vertexX, c->cellX, vx, c->dims.x);
    one_thread_centres(c->vertexY, c->cellY, vy, c->dims.y);
}
#else
extern "C" void ref_initialise_chunk_orig_(const int* chunk, const double* xMin, const double* yMin,
                                           const double* zMin, const double* dx, const double* dy,
                                           const double* dz);

extern "C" void ext_initialise_chunk_(const int* chunk, const double* xMin, const double* yMin, const double* zMin,
                                      const double* dx, const double* dy, const double* dz)
{
    TeaLeafChunk<DEVICE>* c = chunk_at(chunk);
    const std::vector<double> vx = snapshot(c->vertexX), vy = snapshot(c->vertexY), vz = snapshot(c->vertexZ);
    ref_initialise_chunk_orig_(chunk, xMin, yMin, zMin, dx, dy, dz);
    one_thread_centres(c->vertexX, c->cellX, vx, c->dims.x);
    one_thread_centres(c->vertexY, c->cellY, vy, c->dims.y);
    one_thread_centres(c->vertexZ, c->cellZ, vz, c->dims.z);
}
#endif
