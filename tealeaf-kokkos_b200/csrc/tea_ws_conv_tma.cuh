// The warm-start network's convolution fed by the Tensor Memory Accelerator (no counterpart
// in the reference): the row-segment implicit GEMM of k_conv_rows with every operand moved
// by TMA instead of per-thread copies.
//
// A tile is 128 consecutive pixels of one image row (image widths that are multiples of
// 128).  For each of the 3 (2D) or 9 (3D) rows (dz, dy) its taps read, one stage holds
//   A: the row segment x0-1 .. x0+128 of the input, chunk-major: the 16-byte chunk c (8
//      channels) of segment pixel v at byte c * SEG_PITCH * 16 + v * 16, loaded as one 5D
//      TMA box {8 channels, 130 pixels, 1, 1, 1} per chunk from the tensor map of the input
//      (dims channels, W, H, D, n; pixels and rows outside the image, and channels past
//      Cin, arrive as zeros);
//   B: the weights of the row's three taps dx = -1, 0, 1, copied with one bulk copy per tap
//      from a packed copy of the layer's weights that already has the shared-memory layout
//      of the MMA operand (k_pack_weights).
// In the K-major, non-swizzled canonical layout A has its 8-row groups 128 bytes apart (SBO)
// and its K chunks SEG_PITCH * 16 bytes apart (LBO), so the three taps of a row read the
// same segment from 0, 16 and 32 bytes in.
//
// Warp-specialised: one thread of warp 4 issues the copies, up to `stages` stages ahead,
// each stage completing on its "full" mbarrier with the expected byte count; one thread of
// warp 5 issues the tcgen05.mma instructions of a stage once it is full and commits them to
// the stage's "empty" mbarrier (which frees it for the next copy), and after a tile's last
// stage commits to that tile's accumulator mbarrier.  The accumulator is double-buffered in
// tensor memory (tile t in buffer t & 1), so warps 0-3 read tile t for the epilogue of
// k_conv_tc (warp w owns accumulator lanes 32w .. 32w + 31) while the MMAs of tile t + 1
// run; each epilogue warp then arrives on the buffer's "empty" mbarrier.  Every wait is
// bounded: past the limit a role raises the block's abort flag and stops, the others stop
// at their next wait, and the block waits (bounded) for the copies and MMAs it issued,
// frees its tensor memory and reports through the error flag.  The tensor map covers this
// GPU's own buffer only; no copy uses cluster multicast.
#pragma once

#include <cuda.h>

#include "tea_ws_conv.cuh"

namespace tea {
namespace ws {

constexpr int SEG_PITCH = 136;  // 130 pixels used; 136 * 16 bytes is a multiple of 128
constexpr int TMA_MAX_STAGES = 4;

__host__ __device__ constexpr size_t tma_a_bytes(int cin) { return pad1k((size_t)(pad16(cin) / 8) * SEG_PITCH * 16); }
__host__ __device__ constexpr size_t tma_b_tap(int cin, int cout) { return (size_t)pad16(cout) * pad16(cin) * 2; }
__host__ __device__ constexpr size_t tma_stage_bytes(int cin, int cout)
{
    return tma_a_bytes(cin) + pad1k(3 * tma_b_tap(cin, cout));
}
__host__ __device__ constexpr size_t conv_tma_smem_bytes(int cin, int cout, int stages)
{
    return (size_t)stages * tma_stage_bytes(cin, cout) + 1024 + 192;
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void tma_load_5d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3, int c4,
                                            uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, "
        "%6}], [%7];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// The layer's weights w[cout][TAPS][cin] in the MMA's shared-memory layout, per tap
// [np / 8 row groups][kp / 8 chunks][8 rows][8 channels], zero padded to np = pad16(cout)
// rows and kp = pad16(cin) channels: a tap is np * kp contiguous bfloat16 values.
__global__ void k_pack_weights(const bf16* w, bf16* wpk, int cout, int cin)
{
    const int np = pad16(cout), kp = pad16(cin), kc = kp / 8;
    const long total = (long)TAPS * np * kp;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const int e = (int)(i & 7);
        const int j = (int)((i >> 3) & 7);
        long rest = i >> 6;
        const int c = (int)(rest % kc);
        rest /= kc;
        const int gidx = (int)(rest % (np / 8));
        const int t = (int)(rest / (np / 8));
        const int r = gidx * 8 + j, ci = c * 8 + e;
        wpk[i] = (r < cout && ci < cin) ? w[((long)r * TAPS + t) * cin + ci] : __float2bfloat16(0.f);
    }
}

constexpr int TMA_THREADS = 192;  // warps 0-3 epilogue, warp 4 copies, warp 5 MMAs

__global__ void __launch_bounds__(TMA_THREADS) k_conv_tma(ConvArgs a, const bf16* __restrict__ wpk, int stages,
                                                          const __grid_constant__ CUtensorMap tmap)
{
    extern __shared__ __align__(1024) unsigned char s_raw[];
    unsigned char* base = s_raw + ((1024 - (smem_u32(s_raw) & 1023u)) & 1023u);
    const int cin = a.cin, cout = a.cout;
    const int kp = pad16(cin), np = pad16(cout), kchunks = kp / 8;
    const size_t stage_bytes = tma_stage_bytes(cin, cout), a_bytes = tma_a_bytes(cin), b_tap = tma_b_tap(cin, cout);
    uint64_t* full = reinterpret_cast<uint64_t*>(base + (size_t)stages * stage_bytes);
    uint64_t* empty = full + TMA_MAX_STAGES;
    uint64_t* acc_full = empty + TMA_MAX_STAGES;  // [2]: accumulator buffer b complete
    uint64_t* acc_empty = acc_full + 2;           // [2]: accumulator buffer b read by the epilogue
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(acc_empty + 2);
    volatile int* s_abort = reinterpret_cast<volatile int*>(tmem_slot + 1);
    long* s_count = reinterpret_cast<long*>(acc_empty + 3);  // fills issued, fills consumed
    auto sA = [&](int st) { return base + (size_t)st * stage_bytes; };
    auto sB = [&](int st) { return base + (size_t)st * stage_bytes + a_bytes; };

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int ncols = tmem_cols(np);  // one accumulator; two are allocated
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(2 * ncols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int s = 0; s < TMA_MAX_STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&acc_full[b], 1);
            mbar_init(&acc_empty[b], 4);  // one arrival per epilogue warp
        }
        *s_abort = 0;
        s_count[0] = s_count[1] = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmap)) : "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    const long npix = (long)a.n * a.D * a.H * a.W;
    const long ntiles = npix / TC_M;
    const long my_tiles = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    const long nfills = my_tiles * ROW_GROUPS;
    auto give_up = [&]() {
        *s_abort = 1;
        if (a.err) atomicExch(a.err, 1);
    };

    if (warp == 4 && lane == 0) {
        // Copies: fill f into stage f % stages once that stage's MMAs of fill f - stages are done.
        const uint32_t tx_bytes = (uint32_t)(kchunks * 130 * 16 + 3 * b_tap);
        long f = 0;
        for (; f < nfills && !*s_abort; ++f) {
            const int st = (int)(f % stages);
            if (f >= stages && !mbar_wait(&empty[st], (unsigned)(((f / stages) - 1) & 1))) {
                give_up();
                break;
            }
            const long tile = blockIdx.x + (f / ROW_GROUPS) * (long)gridDim.x;
            const int rg = (int)(f % ROW_GROUPS);
            const Pix q = pix_of(tile * TC_M, a.D, a.H, a.W);
            const int dz = WS_3D ? rg / 3 - 1 : 0, dy = rg % 3 - 1;
            mbar_expect_tx(&full[st], tx_bytes);
            for (int c = 0; c < kchunks; ++c)
                tma_load_5d(sA(st) + (size_t)c * SEG_PITCH * 16, &tmap, c * 8, q.x - 1, q.y + dy, q.z + dz,
                            (int)q.img, &full[st]);
            for (int tx = 0; tx < 3; ++tx)
                bulk_load(sB(st) + (size_t)tx * b_tap, wpk + ((size_t)(rg * 3 + tx)) * np * kp, (uint32_t)b_tap,
                          &full[st]);
        }
        s_count[0] = f;
    } else if (warp == 5 && lane == 0) {
        // MMAs: tile tl into accumulator buffer tl & 1, once the epilogue of tile tl - 2 read it.
        const uint32_t idesc = umma_idesc_bf16(TC_M, np);
        const uint32_t lbo_a = SEG_PITCH * 16;       // bytes between the segment's K chunks
        const uint32_t sbo_b = (uint32_t)kp * 16;  // bytes between 8-row groups of the weights
        long f = 0;
        for (long tl = 0; tl < my_tiles && !*s_abort; ++tl) {
            const int ab = (int)(tl & 1);
            if (tl >= 2 && !mbar_wait(&acc_empty[ab], (unsigned)(((tl >> 1) - 1) & 1))) {
                give_up();
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t acc_addr = tmem + (uint32_t)(ab * ncols);
            bool good = true;
            for (int rg = 0; rg < ROW_GROUPS; ++rg, ++f) {
                const int st = (int)(f % stages);
                if (!mbar_wait(&full[st], (unsigned)((f / stages) & 1))) {
                    good = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t a_addr = smem_u32(sA(st)), b_addr = smem_u32(sB(st));
                for (int tx = 0; tx < 3; ++tx) {
                    for (int s = 0; s < kp / 16; ++s) {
                        // Output row m reads segment pixel m + tx (tap dx = tx - 1).
                        const uint64_t da = umma_desc(a_addr + (uint32_t)tx * 16 + (uint32_t)s * 2 * lbo_a, lbo_a, 128);
                        const uint64_t db = umma_desc(b_addr + (uint32_t)(tx * b_tap) + (uint32_t)s * 256, 128, sbo_b);
                        const uint32_t acc = (rg > 0 || tx > 0 || s > 0) ? 1u : 0u;
                        asm volatile(
                            "{\n\t.reg .pred p;\n\t"
                            "setp.ne.b32 p, %4, 0;\n\t"
                            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(acc_addr),
                            "l"(da), "l"(db), "r"(idesc), "r"(acc)
                            : "memory");
                    }
                }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 smem_u32(&empty[st]))
                             : "memory");
            }
            if (!good) {
                give_up();
                break;
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&acc_full[ab]))
                         : "memory");
        }
        s_count[1] = f;
    } else if (warp < 4) {
        // Epilogue: warp w reads accumulator lanes 32w .. 32w + 31 of tile tl's buffer.
        for (long tl = 0; tl < my_tiles && !__any_sync(0xffffffffu, *s_abort); ++tl) {
            const int ab = (int)(tl & 1);
            // The warp decides as one: the accumulator loads below are warp-collective.
            if (!__all_sync(0xffffffffu, mbar_wait(&acc_full[ab], (unsigned)((tl >> 1) & 1)))) {
                if (lane == 0) give_up();
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const long p0 = (blockIdx.x + tl * (long)gridDim.x) * TC_M;
            conv_epilogue(a, tmem + (uint32_t)(ab * ncols), p0, npix, np, warp, lane);
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0)
                asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&acc_empty[ab])) : "memory");
        }
    }
    __syncthreads();
    if (*s_abort && tid == 0) {
        // Copies issued and not consumed, then the MMAs last committed on each stage (bounded).
        const long issued = s_count[0], consumed = s_count[1];
        for (long f = consumed; f < issued; ++f) mbar_wait(&full[f % stages], (unsigned)((f / stages) & 1));
        for (long f = consumed - 1; f >= 0 && f >= consumed - stages; --f)
            mbar_wait(&empty[f % stages], (unsigned)((f / stages) & 1));
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * ncols)
                     : "memory");
    }
}

}  // namespace ws
}  // namespace tea
