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
