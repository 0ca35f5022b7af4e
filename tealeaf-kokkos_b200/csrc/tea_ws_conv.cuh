// Convolutions of the learned warm-start network (no counterpart in the reference).
//
// Activations are bfloat16 channels-last tensors, [n][H][W][C] in the 2D library and
// [n][D][H][W][C] in the 3D one (a 2D image is a volume of depth 1), whose channel
// dimension may be a slice of a wider buffer (channel stride `cs`, first channel `co`), so
// that a decoder's concatenation is written in place.  Weights are stored [Cout][TAPS][Cin]
// (tap t = 3*dy + dx of a 3x3 convolution, t = 9*dz + 3*dy + dx of a 3x3x3 one), bfloat16,
// with float32 biases.  Channel counts are multiples of 8 (16-byte chunks of a pixel's
// channels); the tensor-core kernels pad K and N up to multiples of 16 with zeros.
//
// k_conv_tc is the implicit GEMM on the 5th-generation tensor cores: D[128 pixels x Cout]
// (float32, in tensor memory) += A[128 pixels x Cin] * B[Cout x Cin]^T for each of the
// taps, A gathered from the input shifted by the tap (zero padding) and B the tap's weights,
// both staged by cp.async into shared memory in the K-major, non-swizzled canonical layout
// (8-row x 16-byte core matrices; the descriptor fields follow CUTLASS 4.5's
// cute/arch/mma_sm100_desc.hpp and cute/atom/mma_traits_sm100.hpp).  One thread issues
// tcgen05.mma (kind::f16, M = 128, N = Cout, K = 16 per instruction) and commits them to an
// mbarrier; taps are double-buffered so that the gather of tap t+1 overlaps the MMAs of
// tap t.  The epilogue reads the accumulator with tcgen05.ld (warp w owns TMEM lanes
// 32w..32w+31 = pixels), adds the bias, applies ReLU and/or a ReLU-derivative mask, and
// stores bfloat16.  Every mbarrier wait is bounded: past the limit the kernel records an
// error, stops issuing work, and still frees its tensor memory.
//
// k_conv_ref is the same function on CUDA cores (float32 accumulation): the reference the
// tests hold the tensor-core kernel to.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#ifndef TEA_DIM
#error "compile with -DTEA_DIM=2 or -DTEA_DIM=3"
#endif

namespace tea {
namespace ws {

using bf16 = __nv_bfloat16;

constexpr bool WS_3D = TEA_DIM == 3;
constexpr int TAPS = WS_3D ? 27 : 9;  // 3x3 or 3x3x3 convolutions

__host__ __device__ constexpr int pad16(int c) { return (c + 15) & ~15; }

// Position of pixel p in n images of D x H x W (D = 1 in 2D).
struct Pix {
    int x, y, z;
    long img;
};

__device__ __forceinline__ Pix pix_of(long p, int D, int H, int W)
{
    Pix q;
    q.x = (int)(p % W);
    const long r = p / W;
    q.y = (int)(r % H);
    if (WS_3D) {
        const long s = r / H;
        q.z = (int)(s % D);
        q.img = s / D;
    } else {
        q.z = 0;
        q.img = r / H;
    }
    return q;
}

// The pixel tap t of a convolution reads for output pixel q, or -1 outside the image (the
// zero padding).
__device__ __forceinline__ long tap_src(const Pix& q, int t, int D, int H, int W)
{
    const int sx = q.x + t % 3 - 1, sy = q.y + (t / 3) % 3 - 1, sz = WS_3D ? q.z + t / 9 - 1 : 0;
    if (sx < 0 || sx >= W || sy < 0 || sy >= H || sz < 0 || sz >= D) return -1;
    return ((q.img * D + sz) * (long)H + sy) * W + sx;
}

// A tile's pixel positions, decoded once per tile into shared memory so that the gathers of
// the taps need no divisions: x, y, z of each pixel (x = -1 past the last pixel).
struct TilePix {
    int x, y, z, pad;
};

__device__ __forceinline__ TilePix tile_pix_of(long p, long npix, int D, int H, int W)
{
    TilePix t;
    if (p < npix) {
        const Pix q = pix_of(p, D, H, W);
        t.x = q.x;
        t.y = q.y;
        t.z = q.z;
    } else {
        t.x = -1;
        t.y = t.z = 0;
    }
    t.pad = 0;
    return t;
}

// Whether tap (dz, dy, dx) of pixel q reads a pixel inside the image (false also when q is
// past the last pixel), and the offset of that pixel from q.
__device__ __forceinline__ bool tap_offset(const TilePix& q, int dz, int dy, int dx, int D, int H, int W, long& off)
{
    const int sx = q.x + dx, sy = q.y + dy, sz = q.z + dz;
    off = ((long)dz * H + dy) * W + dx;
    return q.x >= 0 && sx >= 0 && sx < W && sy >= 0 && sy < H && sz >= 0 && sz < D;
}

struct ConvArgs {
    const bf16* x;  // [n][D][H][W][xcs], channels xco .. xco+cin
    int xcs, xco;
    bf16* y;  // [n][D][H][W][ycs], channels yco .. yco+cout
    int ycs, yco;
    const bf16* w;      // [cout][TAPS][cin]
    const float* bias;  // [cout] or null
    const bf16* mask;   // optional: y *= (mask > 0), mask [n][D][H][W][mcs] channels mco..
    int mcs, mco;
    int relu;
    int n, D, H, W, cin, cout;  // D = 1 in 2D
    int* err;  // set to 1 when a bounded wait gave up
};

// ----------------------------------------------------------------------------- reference

__global__ void __launch_bounds__(256) k_conv_ref(ConvArgs a)
{
    const long npix = (long)a.n * a.D * a.H * a.W;
    const long total = npix * a.cout;
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total; idx += (long)gridDim.x * blockDim.x) {
        const int co = (int)(idx % a.cout);
        const long p = idx / a.cout;
        const Pix q = pix_of(p, a.D, a.H, a.W);
        float acc = a.bias ? a.bias[co] : 0.0f;
        for (int t = 0; t < TAPS; ++t) {
            const long sp = tap_src(q, t, a.D, a.H, a.W);
            if (sp < 0) continue;
            const bf16* xp = a.x + sp * a.xcs + a.xco;
            const bf16* wp = a.w + ((long)co * TAPS + t) * a.cin;
            for (int ci = 0; ci < a.cin; ++ci) acc += __bfloat162float(xp[ci]) * __bfloat162float(wp[ci]);
        }
        if (a.relu) acc = fmaxf(acc, 0.0f);
        if (a.mask && !(__bfloat162float(a.mask[p * a.mcs + a.mco + co]) > 0.0f)) acc = 0.0f;
        a.y[p * a.ycs + a.yco + co] = __float2bfloat16(acc);
    }
}

// ----------------------------------------------------------------------------- tcgen05 helpers

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor, K-major without swizzle: LBO = byte distance between the
// two 16-byte K halves of one MMA's K = 16, SBO = byte distance between 8-row groups.
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version of sm_100
    return d;                // base offset 0, layout type 0 (no swizzle)
}

// Instruction descriptor of kind::f16: A, B bfloat16, D float32, both K-major.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int m, int n)
{
    return (1u << 4)                       // D format: F32
         | (1u << 7)                       // A format: BF16
         | (1u << 10)                      // B format: BF16
         | ((uint32_t)(n >> 3) << 17)      // N / 8
         | ((uint32_t)(m >> 4) << 24);     // M / 16
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Bounded wait for the completion of the phase with parity `parity`.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity)
{
    const uint32_t addr = smem_u32(bar);
    for (long it = 0; it < (1L << 24); ++it) {
        uint32_t ok = 0;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(addr), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

__device__ __forceinline__ void cp_async_16z(void* dst, const void* src, bool valid)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)), "l"(src),
                 "r"(valid ? 16 : 0)
                 : "memory");
}

// ----------------------------------------------------------------------------- tensor-core conv

constexpr int TC_THREADS = 128;
constexpr int TC_M = 128;  // pixels per tile

// Shared memory: two stages of A (128 x K) and B (N x K) bfloat16, K and N the channel
// counts padded to multiples of 16, barriers and the tile's pixel positions.
__host__ __device__ constexpr size_t conv_tc_smem_bytes(int cin, int cout)
{
    return 2 * ((size_t)TC_M * pad16(cin) * 2 + (size_t)pad16(cout) * pad16(cin) * 2) + 1024 + 64 +
           TC_M * sizeof(TilePix);
}

__host__ __device__ constexpr int tmem_cols(int cout) { return cout <= 32 ? 32 : (cout <= 64 ? 64 : (cout <= 128 ? 128 : 256)); }

// Epilogue of a 128-pixel tile: warp w reads TMEM lanes 32w..32w+31 (pixels p0 + 32w + lane),
// 16 columns at a time, adds the bias, applies ReLU and/or the mask and stores bfloat16.
__device__ __forceinline__ void conv_epilogue(const ConvArgs& a, uint32_t tmem, long p0, long npix, int np, int warp,
                                              int lane)
{
    const long p = p0 + warp * 32 + lane;
    for (int c0 = 0; c0 < np; c0 += 16) {
        uint32_t r[16];
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
            "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
              "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (p < npix) {
            const int nc = min(16, a.cout - c0);  // real output channels in this group
            __align__(16) bf16 out[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                float v = __uint_as_float(r[j]);
                if (j < nc) {
                    if (a.bias) v += a.bias[c0 + j];
                    if (a.relu) v = fmaxf(v, 0.0f);
                    if (a.mask && !(__bfloat162float(a.mask[p * a.mcs + a.mco + c0 + j]) > 0.0f)) v = 0.0f;
                }
                out[j] = __float2bfloat16(v);
            }
            bf16* dst = a.y + p * a.ycs + a.yco + c0;
            if (nc == 16 && (((uintptr_t)dst) & 15u) == 0) {
                reinterpret_cast<uint4*>(dst)[0] = reinterpret_cast<const uint4*>(out)[0];
                reinterpret_cast<uint4*>(dst)[1] = reinterpret_cast<const uint4*>(out)[1];
            } else {
                for (int j = 0; j < nc; ++j) dst[j] = out[j];
            }
        }
    }
}

// After a block gave up (a bounded wait ran out): wait, bounded, for the MMAs still in
// flight on each stage (the last fill committed there) before their memory is released.
__device__ __forceinline__ void drain_stages(uint64_t* bar, long fill)
{
    for (int s = 0; s < 2; ++s) {
        const long f = ((fill - 1) & 1) == s ? fill - 1 : fill - 2;
        if (f >= 0) mbar_wait(&bar[s], (unsigned)((f >> 1) & 1));
    }
}

__global__ void __launch_bounds__(TC_THREADS) k_conv_tc(ConvArgs a)
{
    extern __shared__ __align__(1024) unsigned char s_raw[];
    // 1024-align the operand area.
    unsigned char* base = s_raw + ((1024 - (smem_u32(s_raw) & 1023u)) & 1023u);
    const int cin = a.cin, cout = a.cout;
    const int kp = pad16(cin), np = pad16(cout);  // K and N of the MMAs (zero padded)
    const size_t a_bytes = (size_t)TC_M * kp * 2, b_bytes = (size_t)np * kp * 2;
    bf16* sA[2] = {reinterpret_cast<bf16*>(base), reinterpret_cast<bf16*>(base + a_bytes + b_bytes)};
    bf16* sB[2] = {reinterpret_cast<bf16*>(base + a_bytes), reinterpret_cast<bf16*>(base + 2 * a_bytes + b_bytes)};
    uint64_t* bar = reinterpret_cast<uint64_t*>(base + 2 * (a_bytes + b_bytes));
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 2);
    int* s_abort = reinterpret_cast<int*>(tmem_slot + 1);
    TilePix* s_pix = reinterpret_cast<TilePix*>(bar + 8);  // 64 bytes past the barriers

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int ncols = tmem_cols(np);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(ncols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        *s_abort = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    const uint32_t idesc = umma_idesc_bf16(TC_M, np);
    const uint32_t sbo = (uint32_t)kp * 16;  // bytes between 8-row groups
    const int kchunks = kp / 8;              // 16-byte chunks per row (those at or past cin are zeros)
    const long npix = (long)a.n * a.D * a.H * a.W;
    const long ntiles = (npix + TC_M - 1) / TC_M;
    long fill = 0;  // fills issued by this CTA (stage = fill & 1)
    bool ok = true;

    for (long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const long p0 = tile * TC_M;
        // Every thread is past the previous tile's gathers (the barrier that ends the tile).
        s_pix[tid] = tile_pix_of(p0 + tid, npix, a.D, a.H, a.W);
        __syncthreads();
        for (int t = 0; t < TAPS && ok; ++t, ++fill) {
            const int st = (int)(fill & 1);
            if (fill >= 2) {
                // The MMAs that last read this stage (fill - 2) must be complete; the decision
                // to give up is made by the whole block at once.
                const bool done = mbar_wait(&bar[st], (unsigned)(((fill - 2) >> 1) & 1));
                if (!__syncthreads_and(done)) {
                    ok = false;
                    break;
                }
            }
            // A: 128 rows (pixels) x kchunks 16-byte chunks.
            const int dz = WS_3D ? t / 9 - 1 : 0, dy = (t / 3) % 3 - 1, dx = t % 3 - 1;
            for (int idx = tid; idx < TC_M * kchunks; idx += TC_THREADS) {
                const int m = idx / kchunks, c = idx - m * kchunks;
                long off;
                const bool valid = tap_offset(s_pix[m], dz, dy, dx, a.D, a.H, a.W, off) && c * 8 < cin;
                const bf16* src = valid ? a.x + (p0 + m + off) * a.xcs + a.xco + c * 8 : a.x;
                bf16* dst = sA[st] + (size_t)(m >> 3) * (sbo / 2) + (size_t)c * 64 + (m & 7) * 8;
                cp_async_16z(dst, src, valid);
            }
            // B: np rows x kchunks chunks of tap t (rows at or past cout are zeros).
            for (int idx = tid; idx < np * kchunks; idx += TC_THREADS) {
                const int r = idx / kchunks, c = idx % kchunks;
                const bool valid = r < cout && c * 8 < cin;
                const bf16* src = valid ? a.w + ((size_t)r * TAPS + t) * cin + c * 8 : a.w;
                bf16* dst = sB[st] + (size_t)(r >> 3) * (sbo / 2) + (size_t)c * 64 + (r & 7) * 8;
                cp_async_16z(dst, src, valid);
            }
            asm volatile("cp.async.wait_all;" ::: "memory");
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();
            if (tid == 0) {
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t a_addr = smem_u32(sA[st]), b_addr = smem_u32(sB[st]);
                for (int s = 0; s < kp / 16; ++s) {
                    const uint64_t da = umma_desc(a_addr + s * 256, 128, sbo);
                    const uint64_t db = umma_desc(b_addr + s * 256, 128, sbo);
                    const uint32_t acc = (t > 0 || s > 0) ? 1u : 0u;
                    asm volatile(
                        "{\n\t.reg .pred p;\n\t"
                        "setp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                        "l"(da), "l"(db), "r"(idesc), "r"(acc)
                        : "memory");
                }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 smem_u32(&bar[st]))
                             : "memory");
            }
        }
        if (!ok) break;
        // All taps issued; wait for the last commit (MMAs complete in order).
        const long last = fill - 1;
        const bool done = mbar_wait(&bar[last & 1], (unsigned)((last >> 1) & 1));
        if (!__syncthreads_and(done)) {
            ok = false;
            break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        conv_epilogue(a, tmem, p0, npix, np, warp, lane);
        // The next tile's MMAs overwrite the accumulator: every lane's reads come first.
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
    }
    if (!ok) {
        *s_abort = 1;
        if (a.err) atomicExch(a.err, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (*s_abort) drain_stages(bar, fill);
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
    }
}

// ----------------------------------------------------------------------------- row-segment conv

// k_conv_rows: the tensor-core convolution for images whose width is a multiple of 128.  A
// tile is 128 consecutive pixels of one image row (x0 .. x0+127).  For each of the 3 (2D) or
// 9 (3D) rows (dz, dy) its taps read, the row segment x0-1 .. x0+128 (130 pixels, zeros
// outside the image) is staged once, chunk-major: the 16-byte chunk c (8 channels) of
// pixel v at byte c * 130 * 16 + v * 16.  In the K-major, non-swizzled canonical layout that
// is a matrix with 8-row groups 128 bytes apart (SBO) and K chunks 2080 bytes apart (LBO),
// so the taps dx = -1, 0, 1 of that row are the same segment read from 0, 16 or 32 bytes in:
// one staged segment serves three taps, where k_conv_tc gathers one 128-pixel slice per
// tap.  The three taps' weights are staged beside it (the canonical layout of k_conv_tc).
// Two stages, one thread issues the MMAs, bounded waits and the epilogue as in k_conv_tc.
constexpr int ROW_SEG = TC_M + 2;
constexpr int ROW_GROUPS = WS_3D ? 9 : 3;

// Operand blocks start on 1024-byte boundaries.
__host__ __device__ constexpr size_t pad1k(size_t b) { return (b + 1023) & ~(size_t)1023; }
__host__ __device__ constexpr size_t rows_a_bytes(int cin) { return pad1k((size_t)ROW_SEG * pad16(cin) * 2); }
__host__ __device__ constexpr size_t rows_b_tap(int cin, int cout) { return pad1k((size_t)pad16(cout) * pad16(cin) * 2); }

__host__ __device__ constexpr size_t conv_rows_smem_bytes(int cin, int cout)
{
    return 2 * (rows_a_bytes(cin) + 3 * rows_b_tap(cin, cout)) + 1024 + 64;
}

__global__ void __launch_bounds__(TC_THREADS) k_conv_rows(ConvArgs a)
{
    extern __shared__ __align__(1024) unsigned char s_raw[];
    unsigned char* base = s_raw + ((1024 - (smem_u32(s_raw) & 1023u)) & 1023u);
    const int cin = a.cin, cout = a.cout;
    const int kp = pad16(cin), np = pad16(cout);
    const size_t a_bytes = rows_a_bytes(cin), b_tap = rows_b_tap(cin, cout), b_bytes = 3 * b_tap;
    bf16* sA[2] = {reinterpret_cast<bf16*>(base), reinterpret_cast<bf16*>(base + a_bytes + b_bytes)};
    bf16* sB[2] = {reinterpret_cast<bf16*>(base + a_bytes), reinterpret_cast<bf16*>(base + 2 * a_bytes + b_bytes)};
    uint64_t* bar = reinterpret_cast<uint64_t*>(base + 2 * (a_bytes + b_bytes));
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 2);
    int* s_abort = reinterpret_cast<int*>(tmem_slot + 1);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int ncols = tmem_cols(np);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(ncols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        *s_abort = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    const uint32_t idesc = umma_idesc_bf16(TC_M, np);
    const uint32_t lbo_a = ROW_SEG * 16;     // bytes between the segment's K chunks
    const uint32_t sbo_b = (uint32_t)kp * 16;  // bytes between 8-row groups of the weights
    const int kchunks = kp / 8;
    const long npix = (long)a.n * a.D * a.H * a.W;
    const long ntiles = npix / TC_M;  // W is a multiple of 128: tiles never straddle rows
    long fill = 0;
    bool ok = true;

    for (long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const long p0 = tile * TC_M;
        const Pix q = pix_of(p0, a.D, a.H, a.W);  // q.x = x0, a multiple of 128
        for (int rg = 0; rg < ROW_GROUPS && ok; ++rg, ++fill) {
            const int st = (int)(fill & 1);
            if (fill >= 2) {
                const bool done = mbar_wait(&bar[st], (unsigned)(((fill - 2) >> 1) & 1));
                if (!__syncthreads_and(done)) {
                    ok = false;
                    break;
                }
            }
            const int dz = WS_3D ? rg / 3 - 1 : 0, dy = rg % 3 - 1;
            const int sy = q.y + dy, sz = q.z + dz;
            const bool row_ok = sy >= 0 && sy < a.H && sz >= 0 && sz < a.D;
            const long row = ((q.img * a.D + sz) * (long)a.H + sy) * a.W;  // first pixel of the source row
            // A: the segment, ROW_SEG pixels x kchunks chunks, chunk-major.
            for (int idx = tid; idx < ROW_SEG * kchunks; idx += TC_THREADS) {
                const int v = idx / kchunks, c = idx - v * kchunks;
                const int sx = q.x - 1 + v;
                const bool valid = row_ok && sx >= 0 && sx < a.W && c * 8 < cin;
                const bf16* src = valid ? a.x + (row + sx) * a.xcs + a.xco + c * 8 : a.x;
                cp_async_16z(sA[st] + (size_t)c * ROW_SEG * 8 + (size_t)v * 8, src, valid);
            }
            // B: the weights of taps (dz, dy, dx = -1, 0, 1): tap index rg * 3 + (dx + 1).
            const int per_tap = np * kchunks;
            for (int idx = tid; idx < 3 * per_tap; idx += TC_THREADS) {
                const int tx = idx / per_tap, rem = idx - tx * per_tap;
                const int r = rem / kchunks, c = rem - r * kchunks;
                const bool valid = r < cout && c * 8 < cin;
                const bf16* src = valid ? a.w + ((size_t)r * TAPS + rg * 3 + tx) * cin + c * 8 : a.w;
                bf16* dst = sB[st] + (size_t)tx * (b_tap / 2) + (size_t)(r >> 3) * (sbo_b / 2) + (size_t)c * 64 +
                            (r & 7) * 8;
                cp_async_16z(dst, src, valid);
            }
            asm volatile("cp.async.wait_all;" ::: "memory");
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();
            if (tid == 0) {
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t a_addr = smem_u32(sA[st]), b_addr = smem_u32(sB[st]);
                for (int tx = 0; tx < 3; ++tx) {
                    for (int s = 0; s < kp / 16; ++s) {
                        // Output row m reads segment pixel m + tx (tap dx = tx - 1).
                        const uint64_t da = umma_desc(a_addr + (uint32_t)tx * 16 + (uint32_t)s * 2 * lbo_a, lbo_a, 128);
                        const uint64_t db = umma_desc(b_addr + (uint32_t)(tx * b_tap) + (uint32_t)s * 256, 128, sbo_b);
                        const uint32_t acc = (rg > 0 || tx > 0 || s > 0) ? 1u : 0u;
                        asm volatile(
                            "{\n\t.reg .pred p;\n\t"
                            "setp.ne.b32 p, %4, 0;\n\t"
                            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                            "l"(da), "l"(db), "r"(idesc), "r"(acc)
                            : "memory");
                    }
                }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 smem_u32(&bar[st]))
                             : "memory");
            }
        }
        if (!ok) break;
        const long last = fill - 1;
        const bool done = mbar_wait(&bar[last & 1], (unsigned)((last >> 1) & 1));
        if (!__syncthreads_and(done)) {
            ok = false;
            break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        conv_epilogue(a, tmem, p0, npix, np, warp, lane);
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
    }
    if (!ok) {
        *s_abort = 1;
        if (a.err) atomicExch(a.err, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (*s_abort) drain_stages(bar, fill);
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
    }
}

// ----------------------------------------------------------------------------- tensor-core weight gradient

// k_wgrad_tc: the weight and bias gradients of a convolution on the tensor cores.  Per
// tap t, gW[co][t][ci] = sum_p gy[p][co] x[p + tap t][ci] is a GEMM with the pixels as its K
// dimension: D[co][ci] (float32, tensor memory) += A[co][p] B[ci][p], A = gy and B = the
// input shifted by the tap.  Both are staged straight from their NHWC rows, whose 16-byte
// chunks hold 8 consecutive channels of one pixel: the MN-major, non-swizzled canonical
// layout (a core matrix is 8 channels x 8 pixels, 128 bytes; core matrices adjacent along
// the channels, SBO = 128 bytes, and groups of 8 pixels LBO bytes apart; descriptor fields
// as CUTLASS 4.5's cute/arch/mma_sm100_desc.hpp and the canonical layouts of
// cute/atom/mma_traits_sm90_gmma.hpp describe them).  M is 128 (rows co >= cout are zero),
// N is cin padded to a multiple of 16, plus 16: the column ci = cin of B is all ones, so
// that D[co][cin] = sum_p gy[p][co] gives the bias gradient (taken from tap 0).  A block owns one tap and a slice of the
// pixels, 64 pixels per stage (four K = 16 MMAs), two stages; one thread issues the MMAs and
// commits them to the stage's mbarrier.  The epilogue reads D with tcgen05.ld and adds it to
// the float32 gradients.  Every wait is bounded, as in k_conv_tc.
constexpr int WT_THREADS = 128;
constexpr int WT_KP = 64;  // pixels per stage

struct WgradArgs {
    const bf16* x;  // [n][D][H][W][xcs], channels xco .. xco+cin
    int xcs, xco;
    const bf16* gy;  // [n][D][H][W][gcs], channels gco .. gco+cout
    int gcs, gco;
    int n, D, H, W, cin, cout;  // D = 1 in 2D
    float* gw;  // [cout][TAPS][cin], accumulated
    float* gb;  // [cout] or null, accumulated
    int* err;
};

__host__ __device__ constexpr size_t wgrad_tc_smem_bytes(int cin)
{
    return 2 * ((size_t)128 * WT_KP * 2 + (size_t)(pad16(cin) + 16) * WT_KP * 2) + 1024 + 64 +
           2 * WT_KP * sizeof(TilePix);
}

__global__ void __launch_bounds__(WT_THREADS) k_wgrad_tc(WgradArgs a)
{
    extern __shared__ __align__(1024) unsigned char s_raw[];
    unsigned char* base = s_raw + ((1024 - (smem_u32(s_raw) & 1023u)) & 1023u);
    const int nb = pad16(a.cin) + 16;  // N: the cin channels, the ones column and zeros
    const size_t a_bytes = (size_t)128 * WT_KP * 2, b_bytes = (size_t)nb * WT_KP * 2;
    bf16* sA[2] = {reinterpret_cast<bf16*>(base), reinterpret_cast<bf16*>(base + a_bytes + b_bytes)};
    bf16* sB[2] = {reinterpret_cast<bf16*>(base + a_bytes), reinterpret_cast<bf16*>(base + 2 * a_bytes + b_bytes)};
    uint64_t* bar = reinterpret_cast<uint64_t*>(base + 2 * (a_bytes + b_bytes));
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 2);
    int* s_abort = reinterpret_cast<int*>(tmem_slot + 1);
    TilePix* s_pix = reinterpret_cast<TilePix*>(bar + 8);  // [stage][WT_KP], 64 bytes past the barriers

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int t = blockIdx.x;  // tap
    const int dz = WS_3D ? t / 9 - 1 : 0, dy = (t / 3) % 3 - 1, dx = t % 3 - 1;
    const int ncols = tmem_cols(nb);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(ncols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        *s_abort = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    const uint32_t idesc = umma_idesc_bf16(128, nb) | (1u << 15) | (1u << 16);  // A and B MN-major
    const uint32_t lbo_a = 128 / 8 * 128, lbo_b = (uint32_t)nb / 8 * 128;    // bytes between pixel groups
    const int gA = 16, gB = nb / 8;                                            // channel groups of 8
    const long npix = (long)a.n * a.D * a.H * a.W;
    const long per = (npix + gridDim.y - 1) / gridDim.y;
    const long pbeg = (long)blockIdx.y * per, pend = min(npix, pbeg + per);
    const long nchunks = pend > pbeg ? (pend - pbeg + WT_KP - 1) / WT_KP : 0;
    long fill = 0;
    bool ok = true;
    for (long ch = 0; ch < nchunks && ok; ++ch, ++fill) {
        const int st = (int)(fill & 1);
        if (fill >= 2) {
            const bool done = mbar_wait(&bar[st], (unsigned)(((fill - 2) >> 1) & 1));
            if (!__syncthreads_and(done)) {
                ok = false;
                break;
            }
        }
        const long p0 = pbeg + ch * WT_KP;
        // The stage's pixel positions (its previous reader, fill - 2, is complete: every
        // thread passed the barrier after that fill's gathers).
        TilePix* spx = s_pix + st * WT_KP;
        if (tid < WT_KP) spx[tid] = tile_pix_of(p0 + tid, pend, a.D, a.H, a.W);
        __syncthreads();
        // A = gy: 16 channel groups (co 0..127; groups at or past cout are zero) x 64 pixels.
        for (int idx = tid; idx < gA * WT_KP; idx += WT_THREADS) {
            const int g = idx % gA, k = idx / gA;
            const long p = p0 + k;
            const bool valid = p < pend && g * 8 < a.cout;
            const bf16* src = valid ? a.gy + p * a.gcs + a.gco + g * 8 : a.gy;
            bf16* dst = sA[st] + ((size_t)(k >> 3) * lbo_a + (size_t)g * 128 + (k & 7) * 16) / 2;
            cp_async_16z(dst, src, valid);
        }
        // B = x shifted by the tap: cin / 8 channel groups, then the ones column and zeros.
        for (int idx = tid; idx < gB * WT_KP; idx += WT_THREADS) {
            const int g = idx % gB, k = idx / gB;
            bf16* dst = sB[st] + ((size_t)(k >> 3) * lbo_b + (size_t)g * 128 + (k & 7) * 16) / 2;
            if (g * 8 < a.cin) {
                long off;
                const bool valid = tap_offset(spx[k], dz, dy, dx, a.D, a.H, a.W, off);
                const bf16* src = valid ? a.x + (p0 + k + off) * a.xcs + a.xco + g * 8 : a.x;
                cp_async_16z(dst, src, valid);
            } else {
                uint4 v = make_uint4(0u, 0u, 0u, 0u);
                if (g * 8 == a.cin) v.x = 0x3F80u;  // bfloat16 1.0 at channel cin
                *reinterpret_cast<uint4*>(dst) = v;
            }
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a_addr = smem_u32(sA[st]), b_addr = smem_u32(sB[st]);
            for (int s = 0; s < WT_KP / 16; ++s) {
                const uint64_t da = umma_desc(a_addr + s * 2 * lbo_a, lbo_a, 128);
                const uint64_t db = umma_desc(b_addr + s * 2 * lbo_b, lbo_b, 128);
                const uint32_t acc = (fill > 0 || s > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                    "l"(da), "l"(db), "r"(idesc), "r"(acc)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&bar[st]))
                         : "memory");
        }
    }
    if (ok && fill > 0) {
        const long last = fill - 1;
        const bool done = mbar_wait(&bar[last & 1], (unsigned)((last >> 1) & 1));
        if (!__syncthreads_and(done)) ok = false;
    }
    if (ok && fill > 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        // Warp w reads TMEM lanes 32w..32w+31 (rows co), 16 columns (ci) at a time.
        const int co = warp * 32 + lane;
        for (int c0 = 0; c0 < nb; c0 += 16) {
            uint32_t r[16];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (co < a.cout) {
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int ci = c0 + j;
                    const float v = __uint_as_float(r[j]);
                    if (ci < a.cin) atomicAdd(&a.gw[((long)co * TAPS + t) * a.cin + ci], v);
                    else if (ci == a.cin && t == 0 && a.gb) atomicAdd(&a.gb[co], v);
                }
            }
        }
    }
    if (!ok) {
        *s_abort = 1;
        if (a.err) atomicExch(a.err, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (*s_abort) drain_stages(bar, fill);
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
    }
}

}  // namespace ws
}  // namespace tea
