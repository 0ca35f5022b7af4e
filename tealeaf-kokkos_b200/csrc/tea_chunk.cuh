// Host-side chunk state of the TeaLeaf B200 library and the small utilities every entry
// point uses (status recording, launch sizing).  One Chunk replaces the reference's
// TeaLeafChunk<Device> (tealeaf_2d/ext_chunk.hpp:16-73, tealeaf_3d/ext_chunk.hpp): the
// same arrays, held in HBM in the pitched layout of tea_common.cuh.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <string>
#include <vector>

#include "tea_common.cuh"

namespace tea {

// Fields held per chunk; 1..15 match the field ids of include/tea_b200.h.
enum FieldId {
    F_DENSITY = 1, F_ENERGY0, F_ENERGY1, F_U, F_P, F_SD, F_U0, F_R, F_W, F_Z, F_MI,
    F_KX, F_KY, F_KZ, F_VOLUME, F_COUNT = 16
};

struct Fields {
    double *density, *energy0, *energy, *u, *u0, *p, *r, *mi, *w, *z, *kx, *ky, *kz, *sd, *volume;
};

// An iteration box [k0,k1) x [j0,j1) x [i0,i1) over padded indices, walked in tiles.
struct Box {
    int k0, k1, j0, j1, i0, i1;
    int tx, ty;
    long ntiles;
};

inline Box make_box(int k0, int k1, int j0, int j1, int i0, int i1)
{
    Box b;
    b.k0 = k0; b.k1 = k1; b.j0 = j0; b.j1 = j1; b.i0 = i0; b.i1 = i1;
    b.tx = k1 > k0 ? (k1 - k0 + TILE_X - 1) / TILE_X : 0;
    b.ty = j1 > j0 ? (j1 - j0 + TILE_Y - 1) / TILE_Y : 0;
    b.ntiles = (long)b.tx * b.ty * (i1 > i0 ? (i1 - i0) : 0);
    return b;
}

template <class F>
__device__ __forceinline__ void walk(const Box& b, F&& f)
{
    for (long t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
        const int tx = (int)(t % b.tx);
        const long rest = t / b.tx;
        const int ty = (int)(rest % b.ty);
        const int tz = (int)(rest / b.ty);
        const int kk = b.k0 + tx * TILE_X + (int)threadIdx.x;
        const int jj = b.j0 + ty * TILE_Y + (int)threadIdx.y;
        const int ii = b.i0 + tz;
        if (kk < b.k1 && jj < b.j1) f(kk, jj, ii);
    }
}

struct Chunk {
    Geom g;
    Box inner, full, one, skew;
    int rank = 0;
    double dx = 0, dy = 0, dz = 0, theta = 0;
    int preconditioner = 0;
    Fields f{};
    double* alloc[F_COUNT] = {};
    size_t field_elems = 0;  // doubles per allocation (lead pad included)
    // Coordinates: tiny, computed on the host (see ext_initialise_chunk_), mirrored.
    std::vector<double> vx, vy, vz, cx, cy, cz;
    double *d_vx = nullptr, *d_vy = nullptr, *d_vz = nullptr, *d_cx = nullptr, *d_cy = nullptr,
           *d_cz = nullptr;
    // Chebyshev / PPCG coefficients (host copy; the kernels take them by value).
    std::vector<double> h_alphas, h_betas;
    cudaStream_t stream = nullptr;
    RedScratch red{};
    double* h_out = nullptr;  // mapped pinned host memory for reduction results
    double* d_out = nullptr;  // its device alias
    int grid_blocks = 0;      // blocks for grid-stride per-call kernels
    int device = 0;
    void* fused = nullptr;    // whole-solve state (tea_fused.cuh)
    void* ws = nullptr;       // attached warm-start network (tea_warmstart.cu), not owned
    int ws_reject_streak = 0; // consecutive timesteps whose guess was rejected
    int ws_skip = 0;          // timesteps left to solve without a guess (back-off)
    long long h2d_bytes = 0;  // host<->device bytes moved for this chunk (inputs, results)
    long long d2h_bytes = 0;
};

// ------------------------------------------------------------------ status

struct StatusStore {
    int status = 0;
    std::string message;
};

inline StatusStore& status_store()
{
    static StatusStore s;
    return s;
}

inline void set_status(int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    StatusStore& s = status_store();
    if (s.status == 0 || code == 3 /* CUDA errors win */) {
        s.status = code;
        s.message = buf;
    }
    std::fprintf(stderr, "tea_b200: %s\n", buf);
}

#define TEA_CK(call)                                                                               \
    do {                                                                                           \
        cudaError_t tea_ck_e = (call);                                                             \
        if (tea_ck_e != cudaSuccess)                                                               \
            ::tea::set_status(3, "%s failed at %s:%d: %s", #call, __FILE__, __LINE__,              \
                              cudaGetErrorString(tea_ck_e));                                       \
    } while (0)

// Host<->device copy ordered on `s` and complete on return.  The library's streams are
// non-blocking, so a plain cudaMemcpy (legacy stream) is not ordered with their kernels,
// and from pageable memory it may return before the data has landed.
inline cudaError_t copy_on(cudaStream_t s, void* dst, const void* src, size_t bytes, cudaMemcpyKind kind)
{
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, kind, s);
    return e != cudaSuccess ? e : cudaStreamSynchronize(s);
}

inline int launch_blocks(const Chunk* c, long ntiles)
{
    long b = ntiles < c->grid_blocks ? ntiles : c->grid_blocks;
    return b < 1 ? 1 : (int)b;
}

}  // namespace tea
