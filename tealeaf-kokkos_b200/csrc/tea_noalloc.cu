// tea_2norm_noalloc_: the 2-norm of ext_calculate_2norm_ over an array the caller owns,
// without allocating any device memory.
//
// Who needs it: a caller that keeps its fields in its own device buffers and whose
// device memory is handed out by its own pool allocator (a framework that reserves most
// of HBM up front, or a Fortran/OpenACC code that manages its arrays itself) cannot let a
// library call cudaMalloc: once the pool holds the memory the allocation fails, and even
// when it succeeds it fragments memory the caller accounts for.  Such a caller also has
// no chunk of this library to point at.  This entry point takes the caller's array and
// the caller's output slot and uses, for its reduction scratch (the per-block partial
// sums and the arrival counter of the single-pass grid reduction), one file-scope static
// device array of fixed size instead of allocated memory.
//
// The static array exists once per GPU that loads the library and stays until the
// process exits.  Every call shares it and it keeps the last call's contents: the
// counter is cleared at the start of each call, and calls whose kernels overlap on the
// GPU (different streams, or different host threads without ordering) race on it.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/tea_b200.h"
#include "tea_chunk.cuh"

#define TEA_EXPORT extern "C" __attribute__((visibility("default")))

namespace tea {
namespace {

constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocCellsPerThread = 8;
constexpr int kNoAllocCellsPerBlock = kNoAllocThreads * kNoAllocCellsPerThread;  // 2048
constexpr int kNoAllocMaxBlocks = 8192;
// The largest inner domain one call accepts: 8192 blocks x 2048 cells = 16,777,216 cells
// (4096 x 4096, or 256^3).
constexpr long long kNoAllocMaxCells = (long long)kNoAllocMaxBlocks * kNoAllocCellsPerBlock;

struct NoAllocScratch {
    DD partials[kNoAllocMaxBlocks];  // one double-double partial sum per block
    unsigned int counter;            // blocks arrived; must be 0 when a launch starts
};

// 128 KB + the counter, per device.
static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
NoAllocScratch* g_scratch_addr[kMaxDevices] = {};

// Calculate2Norm (tealeaf_2d/ext_solver_methods.hpp:70-92) over the inner domain of a flat
// padded array (x fastest, HALO_PAD = 2 on every side), one block per 2048 consecutive
// inner cells; sums in double-double.  The last block to arrive merges the block partials
// in a fixed order (lane-strided, then a butterfly) and rounds once.  That order is not
// ext_calculate_2norm_'s, so the two agree because the double-double sum carries far more
// bits than the result keeps, not by construction: they can differ in the last bit only
// where the exact sum lies within about n * 2^-106 of a rounding boundary.
__global__ void __launch_bounds__(kNoAllocThreads) k_2norm_noalloc(const double* __restrict__ field, int nx, int ny,
                                                                   long long ncells, NoAllocScratch* scratch,
                                                                   double* out)
{
    const long X = nx + 2 * HALO_PAD, Y = ny + 2 * HALO_PAD;
    DD acc;
    acc.hi = acc.lo = 0.0;
    const long long base = (long long)blockIdx.x * kNoAllocCellsPerBlock;
    for (int k = 0; k < kNoAllocCellsPerThread; ++k) {
        const long long t = base + (long long)k * kNoAllocThreads + threadIdx.x;
        if (t < ncells) {
            const long kk = HALO_PAD + (long)(t % nx);
            const long rest = (long)(t / nx);
            const long jj = HALO_PAD + rest % ny;
            const long ii = rest / ny + (DIM == 3 ? HALO_PAD : 0);
            const double v = field[kk + X * (jj + Y * ii)];
            dd_add(acc, v * v);
        }
    }
    // Warp, then block, merge in a fixed order.
    for (int o = 16; o > 0; o >>= 1) {
        DD b;
        b.hi = __shfl_xor_sync(0xffffffffu, acc.hi, o);
        b.lo = __shfl_xor_sync(0xffffffffu, acc.lo, o);
        acc = dd_merge(acc, b);
    }
    __shared__ DD s_warp[kNoAllocThreads / 32];
    __shared__ bool s_last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) s_warp[warp] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        DD b;
        b.hi = b.lo = 0.0;
        for (int w = 0; w < kNoAllocThreads / 32; ++w) b = dd_merge(b, s_warp[w]);
        scratch->partials[blockIdx.x] = b;
        __threadfence();
        s_last = atomicAdd(&scratch->counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last || warp != 0) return;
    __threadfence();
    DD b;
    b.hi = b.lo = 0.0;
    for (int blk = lane; blk < (int)gridDim.x; blk += 32) {
        DD p;
        p.hi = __ldcg(&scratch->partials[blk].hi);
        p.lo = __ldcg(&scratch->partials[blk].lo);
        b = dd_merge(b, p);
    }
    for (int o = 16; o > 0; o >>= 1) {
        DD c;
        c.hi = __shfl_xor_sync(0xffffffffu, b.hi, o);
        c.lo = __shfl_xor_sync(0xffffffffu, b.lo, o);
        b = dd_merge(b, c);
    }
    if (lane == 0) {
        *out = dd_value(b);
        scratch->counter = 0u;
    }
}

// Device address of the static scratch on the current device, looked up once per device
// (on the first call there).  The cached address assumes the device is not reset while the
// library is loaded: cudaDeviceReset recreates the module, and the array with it.
NoAllocScratch* scratch_for_current_device(int* status)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        set_status(TEA_ERR_CUDA, "tea_2norm_noalloc_: cudaGetDevice: %s", cudaGetErrorString(e));
        *status = TEA_ERR_CUDA;
        return nullptr;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        set_status(TEA_ERR_BAD_ARGUMENT, "tea_2norm_noalloc_: device %d is beyond the %d devices it serves", dev,
                   kMaxDevices);
        *status = TEA_ERR_BAD_ARGUMENT;
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[dev]) {
        void* ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr) {
            set_status(TEA_ERR_CUDA, "tea_2norm_noalloc_: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
            *status = TEA_ERR_CUDA;
            return nullptr;
        }
        g_scratch_addr[dev] = static_cast<NoAllocScratch*>(ptr);
    }
    return g_scratch_addr[dev];
}

}  // namespace
}  // namespace tea

using namespace tea;

TEA_EXPORT int tea_2norm_noalloc_(const double* field, const int* nx, const int* ny, const int* nz, double* norm,
                                  void* stream)
{
    const int z = (DIM == 3) ? *nz : 1;
    if (*nx < 1 || *ny < 1 || z < 1 || !field || !norm) {
        set_status(TEA_ERR_BAD_ARGUMENT, "tea_2norm_noalloc_: invalid arguments");
        return TEA_ERR_BAD_ARGUMENT;
    }
    const long long ncells = (long long)*nx * *ny * z;
    if (ncells > kNoAllocMaxCells) {
        set_status(TEA_ERR_BAD_ARGUMENT,
                   "tea_2norm_noalloc_: %lld inner cells exceed the maximum of %lld that its static scratch serves",
                   ncells, kNoAllocMaxCells);
        return TEA_ERR_BAD_ARGUMENT;
    }
    int status = TEA_OK;
    NoAllocScratch* scratch = scratch_for_current_device(&status);
    if (!scratch) return status;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(&scratch->counter, 0, sizeof(unsigned int), s);
    if (e == cudaSuccess) {
        const int blocks = (int)((ncells + kNoAllocCellsPerBlock - 1) / kNoAllocCellsPerBlock);
        k_2norm_noalloc<<<blocks, kNoAllocThreads, 0, s>>>(field, *nx, *ny, ncells, scratch, norm);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        set_status(TEA_ERR_CUDA, "tea_2norm_noalloc_: %s", cudaGetErrorString(e));
        return TEA_ERR_CUDA;
    }
    return TEA_OK;
}
