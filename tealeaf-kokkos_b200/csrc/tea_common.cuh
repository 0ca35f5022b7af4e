// Shared device-side infrastructure of the TeaLeaf B200 library: the field layout in
// HBM, the tile walk used by the per-call kernels, and the deterministic double-double
// grid reduction.  Compiled into both libtea2d_b200.so and libtea3d_b200.so
// (-DTEA_DIM=2 / -DTEA_DIM=3).  Build with -fmad=false: every multiply and add is
// rounded separately, exactly as the reference's C++ (and the oracle) evaluate them.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#ifndef TEA_DIM
#error "compile with -DTEA_DIM=2 or -DTEA_DIM=3"
#endif

namespace tea {

constexpr int DIM = TEA_DIM;
constexpr int HALO_PAD = 2;
// Field layout: element (kk, jj, ii) of a padded array (kk in [0, nx+4) etc., the
// reference's flat index kk + jj*X + ii*X*Y) lives at f[kk + jj*pitch + ii*page] with
// pitch = roundup(nx+4, 32) doubles and f = allocation + kLeadPad, so the first inner
// cell of every row (kk = 2) starts on a 256-byte boundary.
constexpr int kLeadPad = 30;
constexpr int kPitchAlign = 32;

// Per-call kernels walk the inner domain in 32 x 8 tiles (one z-plane per tile in 3D).
constexpr int TILE_X = 32;
constexpr int TILE_Y = 8;
constexpr int BLOCK = TILE_X * TILE_Y;
constexpr int MAX_RED = 4;  // values per reduction (field summary needs 4)

struct Geom {
    int nx, ny, nz;     // inner cells (nz = 1 in 2D)
    int X, Y, Z;        // padded extents (Z = 1 in 2D)
    long pitch, page;   // elements
    int tiles_x, tiles_y;
    long tiles_inner;   // tiles covering the inner domain
    int ftiles_x, ftiles_y;
    long tiles_full;    // tiles covering the whole padded array
};

__host__ __device__ inline long fidx(const Geom& g, int kk, int jj, int ii)
{
    return (long)kk + (long)jj * g.pitch + (long)ii * g.page;
}

// ------------------------------------------------------------------ double-double sums

struct DD {
    double hi, lo;
};

// Knuth's TwoSum accumulation (cascaded summation): hi + lo carries the running sum to
// about twice the working precision, so the final hi + lo is the correctly rounded sum
// except within ~n*2^-106 of a rounding boundary, independent of the summation order.
__device__ __forceinline__ void dd_add(DD& a, double x)
{
    const double s = a.hi + x;
    const double bp = s - a.hi;
    const double e = (a.hi - (s - bp)) + (x - bp);
    a.hi = s;
    a.lo = a.lo + e;
}

__device__ __forceinline__ DD dd_merge(DD a, DD b)
{
    const double s = a.hi + b.hi;
    const double bp = s - a.hi;
    const double e = (a.hi - (s - bp)) + (b.hi - bp);
    DD r;
    r.hi = s;
    r.lo = (a.lo + b.lo) + e;
    return r;
}

__device__ __forceinline__ double dd_value(DD a) { return a.hi + a.lo; }

template <int NV>
struct DDVec {
    DD v[NV];
    __device__ __forceinline__ void zero()
    {
#pragma unroll
        for (int k = 0; k < NV; ++k) v[k].hi = v[k].lo = 0.0;
    }
};

// Grid reduction scratch: one DD per value per block, and an arrival counter.
struct RedScratch {
    DD* partials;           // [max_blocks * MAX_RED]
    unsigned int* counter;  // reset to 0 by the last block
    int max_blocks;
};

template <int NV>
__device__ __forceinline__ void warp_merge(DDVec<NV>& a)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            DD b;
            b.hi = __shfl_xor_sync(0xffffffffu, a.v[k].hi, o);
            b.lo = __shfl_xor_sync(0xffffffffu, a.v[k].lo, o);
            a.v[k] = dd_merge(a.v[k], b);
        }
    }
}

// Last block of a grid reduction: every thread merges a strided share of the block
// partials (up to four loads in flight per thread), then a fixed-order warp merge and a
// merge of the warps in order through `s` (nwarps x NV, shared).  The order depends only on
// the grid and block sizes.  Called by every thread of the last block; the result is valid
// in thread 0.
template <int NV>
__device__ __forceinline__ DDVec<NV> merge_partials(const RedScratch& rs, DD* s, int tid, int nthreads)
{
    const int lane = tid & 31, warp = tid >> 5, nwarps = nthreads >> 5;
    DDVec<NV> b;
    b.zero();
    const int nblk = (int)gridDim.x;
    for (int blk0 = tid; blk0 < nblk; blk0 += 4 * nthreads) {
        DD p[4][NV];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int blk = blk0 + u * nthreads;
#pragma unroll
            for (int k = 0; k < NV; ++k) {
                p[u][k].hi = blk < nblk ? __ldcg(&rs.partials[(long)blk * MAX_RED + k].hi) : 0.0;
                p[u][k].lo = blk < nblk ? __ldcg(&rs.partials[(long)blk * MAX_RED + k].lo) : 0.0;
            }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int k = 0; k < NV; ++k) b.v[k] = dd_merge(b.v[k], p[u][k]);
    }
    warp_merge<NV>(b);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) s[warp * NV + k] = b.v[k];
    }
    __syncthreads();
    if (tid == 0) {
        b.zero();
        for (int w = 0; w < nwarps; ++w)
#pragma unroll
            for (int k = 0; k < NV; ++k) b.v[k] = dd_merge(b.v[k], s[w * NV + k]);
    }
    return b;
}

// Block-reduce `acc`, then the last block to arrive merges every block's partial in
// block order and writes the rounded results to out[0..NV).  Deterministic for a given
// grid size; no block waits on another.  Must be called by every thread of the block.
template <int NV>
__device__ void grid_reduce(DDVec<NV> acc, const RedScratch& rs, double* out)
{
    __shared__ DD s_warp[BLOCK / 32][NV];
    __shared__ bool s_last;
    const int lane = threadIdx.x & 31;
    const int tid = threadIdx.x + threadIdx.y * blockDim.x;
    const int warp = tid >> 5;
    const int nwarps = (blockDim.x * blockDim.y) >> 5;
    warp_merge<NV>(acc);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) s_warp[warp][k] = acc.v[k];
    }
    __syncthreads();
    if (tid == 0) {
        DDVec<NV> b;
        b.zero();
        for (int w = 0; w < nwarps; ++w)
#pragma unroll
            for (int k = 0; k < NV; ++k) b.v[k] = dd_merge(b.v[k], s_warp[w][k]);
#pragma unroll
        for (int k = 0; k < NV; ++k) rs.partials[(long)blockIdx.x * MAX_RED + k] = b.v[k];
        __threadfence();
        const unsigned int prev = atomicAdd(rs.counter, 1u);
        s_last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (!s_last) return;
    // Last block: every thread merges a share of the partials (fixed order).
    __threadfence();
    const DDVec<NV> b = merge_partials<NV>(rs, &s_warp[0][0], tid, nwarps * 32);
    if (tid == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) out[k] = dd_value(b.v[k]);
        *rs.counter = 0u;
    }
}

// As grid_reduce, but the last block's lane 0 hands the rounded values to `f` (the
// solver's scalar recurrence and loop control run there, with every other block done).
template <int NV, class F>
__device__ void grid_reduce_then(DDVec<NV> acc, const RedScratch& rs, F&& f)
{
    __shared__ DD s_warp2[32][NV];
    __shared__ bool s_last2;
    const int lane = threadIdx.x & 31;
    const int tid = threadIdx.x + threadIdx.y * blockDim.x;
    const int warp = tid >> 5;
    const int nwarps = (blockDim.x * blockDim.y) >> 5;
    warp_merge<NV>(acc);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) s_warp2[warp][k] = acc.v[k];
    }
    __syncthreads();
    if (tid == 0) {
        DDVec<NV> b;
        b.zero();
        for (int w = 0; w < nwarps; ++w)
#pragma unroll
            for (int k = 0; k < NV; ++k) b.v[k] = dd_merge(b.v[k], s_warp2[w][k]);
#pragma unroll
        for (int k = 0; k < NV; ++k) rs.partials[(long)blockIdx.x * MAX_RED + k] = b.v[k];
        __threadfence();
        const unsigned int prev = atomicAdd(rs.counter, 1u);
        s_last2 = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (!s_last2) return;
    __threadfence();
    const DDVec<NV> b = merge_partials<NV>(rs, &s_warp2[0][0], tid, nwarps * 32);
    if (tid == 0) {
        double vals[NV];
#pragma unroll
        for (int k = 0; k < NV; ++k) vals[k] = dd_value(b.v[k]);
        *rs.counter = 0u;
        f(vals);
    }
}

}  // namespace tea
