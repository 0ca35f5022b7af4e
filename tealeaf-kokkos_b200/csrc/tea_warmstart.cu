// Learned warm start of the implicit solve (no counterpart in the reference).
//
// A small U-Net (tea_ws_conv.cuh, tea_ws_kernels.cuh; the numpy restatement is
// oracle/warmstart_oracle.py) predicts the timestep increment du = u(n+1) - u0 from the
// step's inputs u0 = density * energy, density, Kx, Ky (and Kz) -- through r0 = u0 - A u0, the
// residual of the plain start (A du = r0, so the network learns an approximate inverse of
// the operator; normalising r0 and du by max |r0| keeps every timestep at unit scale).  The solve starts from
// u0 + du when that guess has a smaller FP64 initial residual than u0 itself, and
// converges to the same tolerance either way, so no network error survives.  Training
// pairs are recorded from the solver's own timesteps (tea_ws_record_), the network is
// trained on the GPU by this file's forward and backward kernels (bfloat16 storage,
// float32 accumulation, Adam on float32 master weights) and attached to a chunk
// (tea_ws_attach_), whose whole-solve calls then warm-start from it.  The 2D library's
// network is built from 3x3 convolutions and 2x2 pooling over [ny][nx] images, the 3D
// library's from 3x3x3 convolutions and 2x2x2 pooling over [nz][ny][nx] volumes; a 2D image
// is handled as a volume of depth 1 throughout.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <random>
#include <vector>

#include "../../include/tea_b200.h"
#include "tea_chunk.cuh"
#include "tea_common.cuh"
#include "tea_ws_conv_tma.cuh"
#include "tea_ws_kernels.cuh"

#include <cudaTypedefs.h>

#define TEA_EXPORT extern "C" __attribute__((visibility("default")))

namespace tea {

Chunk* get_chunk(const int* chunk);

namespace ws {

constexpr int IN_PAD = 16;  // network input channels as stored (the features, zero padding)
constexpr int N_FEAT = WS_3D ? 5 : 4;

// ----------------------------------------------------------------------------- chunk <-> features

// Inner cell i (x fastest, then y, then z) of the chunk: its padded indices and field offset.
struct Cell {
    int kk, jj, ii;
    long f;
};

__device__ __forceinline__ Cell cell_of(const Geom& g, long i)
{
    Cell c;
    c.kk = HALO_PAD + (int)(i % g.nx);
    const long r = i / g.nx;
    c.jj = HALO_PAD + (int)(r % g.ny);
    c.ii = WS_3D ? HALO_PAD + (int)(r / g.ny) : 0;
    c.f = fidx(g, c.kk, c.jj, c.ii);
    return c;
}

__host__ __device__ inline long inner_cells(const Geom& g) { return (long)g.nx * g.ny * (WS_3D ? g.nz : 1); }

// A v at inner cell c with the neighbours outside the domain taken as the cell itself (the
// reflected halo), in the operand order of the solver's operator.  With `no_flux` the
// coefficients of the domain's outer faces are taken as zero instead (used by the
// smoothing sweeps; the reflection gives the same product, since v_nb = v there).
__device__ __forceinline__ double apply_a_cell(const Geom& g, const Cell& c, const double* v, const double* kx,
                                               const double* ky, const double* kz, bool no_flux, double* diag)
{
    const int xlast = g.X - HALO_PAD - 1, ylast = g.Y - HALO_PAD - 1, zlast = g.Z - HALO_PAD - 1;
    const long f = c.f;
    const double u = v[f];
    const double xm = c.kk > HALO_PAD ? v[f - 1] : u, xp = c.kk < xlast ? v[f + 1] : u;
    const double ym = c.jj > HALO_PAD ? v[f - g.pitch] : u, yp = c.jj < ylast ? v[f + g.pitch] : u;
    double kx0 = kx[f], kx1 = kx[f + 1], ky0 = ky[f], ky1 = ky[f + g.pitch];
    if (no_flux) {
        if (c.kk == HALO_PAD) kx0 = 0.0;
        if (c.kk == xlast) kx1 = 0.0;
        if (c.jj == HALO_PAD) ky0 = 0.0;
        if (c.jj == ylast) ky1 = 0.0;
    }
    if (!WS_3D) {
        const double d = 1.0 + (kx1 + kx0) + (ky1 + ky0);
        if (diag) *diag = d;
        return d * u - (kx1 * xp + kx0 * xm) - (ky1 * yp + ky0 * ym);
    }
    const double zm = c.ii > HALO_PAD ? v[f - g.page] : u, zp = c.ii < zlast ? v[f + g.page] : u;
    double kz0 = kz[f], kz1 = kz[f + g.page];
    if (no_flux) {
        if (c.ii == HALO_PAD) kz0 = 0.0;
        if (c.ii == zlast) kz1 = 0.0;
    }
    const double d = 1.0 + (kx1 + kx0) + (ky1 + ky0) + (kz1 + kz0);
    if (diag) *diag = d;
    return d * u - (kx1 * xp + kx0 * xm) - (ky1 * yp + ky0 * ym) - (kz1 * zp + kz0 * zm);
}

// The plain start's residual r0 = u0 - A u0 (FP64) over the inner cells, [nz][ny][nx]; the
// neighbours outside the domain are the reflected cells, as the halo update makes them.
__global__ void k_r0(Geom g, const double* u0, const double* kx, const double* ky, const double* kz, double* r0)
{
    const long n = inner_cells(g);
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const Cell c = cell_of(g, i);
        r0[i] = u0[c.f] - apply_a_cell(g, c, u0, kx, ky, kz, false, nullptr);
    }
}

// Largest |v| over n values: per-block maxima (partial), then one block (k_absmax_final).
__global__ void k_absmax(const double* v, long n, double* partial)
{
    __shared__ double s[256];
    double m = 0.0;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        m = fmax(m, fabs(v[i]));
    s[threadIdx.x] = m;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) s[threadIdx.x] = fmax(s[threadIdx.x], s[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = s[0];
}

__global__ void k_absmax_final(const double* partial, int n, double* out)
{
    __shared__ double s[256];
    double m = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) m = fmax(m, partial[i]);
    s[threadIdx.x] = m;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) s[threadIdx.x] = fmax(s[threadIdx.x], s[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = s[0] > 0.0 ? s[0] : 1.0;
}

// Network input of the chunk's timestep: [nz][ny][nx][IN_PAD] bfloat16, channels r0 / scale
// (scale = max |r0|), log10(density) / 2, log10(1 + Kx) / 4, log10(1 + Ky) / 4 (and
// log10(1 + Kz) / 4), then zeros.
__global__ void k_features(Geom g, const double* r0, const double* dens, const double* kx, const double* ky,
                           const double* kz, const double* scale, bf16* x)
{
    const long n = inner_cells(g);
    const double inv = 1.0 / scale[0];
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const long f = cell_of(g, i).f;
        __align__(16) bf16 v[IN_PAD];
        v[0] = __float2bfloat16((float)(r0[i] * inv));
        v[1] = __float2bfloat16((float)(log10(dens[f]) * 0.5));
        v[2] = __float2bfloat16((float)(log10(1.0 + kx[f]) * 0.25));
        v[3] = __float2bfloat16((float)(log10(1.0 + ky[f]) * 0.25));
        if (WS_3D) v[4] = __float2bfloat16((float)(log10(1.0 + kz[f]) * 0.25));
        for (int c = N_FEAT; c < IN_PAD; ++c) v[c] = __float2bfloat16(0.f);
        uint4* dst = reinterpret_cast<uint4*>(x + i * IN_PAD);
        dst[0] = reinterpret_cast<const uint4*>(v)[0];
        dst[1] = reinterpret_cast<const uint4*>(v)[1];
    }
}

// A recorded pair: the features, the target (u - u0) / scale (scale = max |r0|), and the
// cell's face coefficients (Kx, Ky[, Kz]) for the residual loss.
__global__ void k_record(Geom g, const bf16* x, const double* u, const double* u0, const double* kx, const double* ky,
                         const double* kz, const double* scale, bf16* feat, float* tgt, float* kxy)
{
    const long n = inner_cells(g);
    const double inv = 1.0 / scale[0];
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const long f = cell_of(g, i).f;
        for (int c = 0; c < N_FEAT; ++c) feat[i * N_FEAT + c] = x[i * IN_PAD + c];
        tgt[i] = (float)((u[f] - u0[f]) * inv);
        kxy[NK * i] = (float)kx[f];
        kxy[NK * i + 1] = (float)ky[f];
        if (WS_3D) kxy[NK * i + 2] = (float)kz[f];
    }
}

// One damped Jacobi sweep of the guess in FP64: out = u + omega (u0 - A u) / diag(A), no
// flux through the domain's faces (the reflected neighbours).
__global__ void k_ws_smooth(Geom g, const double* u, const double* u0, const double* kx, const double* ky,
                            const double* kz, double* out)
{
    const long n = inner_cells(g);
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const Cell c = cell_of(g, i);
        double d = 1.0;
        const double au = apply_a_cell(g, c, u, kx, ky, kz, true, &d);
        out[c.f] = u[c.f] + (double)WS_OMEGA * (u0[c.f] - au) / d;
    }
}

// u = u0 + y * scale over the inner cells.
__global__ void k_apply_guess(Geom g, const float* y, const double* u0, const double* scale, double inv_out,
                              double* u)
{
    const long n = inner_cells(g);
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const long f = cell_of(g, i).f;
        u[f] = u0[f] + (double)y[i] * inv_out * scale[0];
    }
}

struct Crop {
    const bf16* feat;
    const float* tgt;
    const float* kk;
    int H, W, z0, y0, x0;  // source height and width, crop origin (z0 = 0 in 2D)
};

// Training batch: b crops of s x s (x s in 3D) cells from recorded pairs.
__global__ void k_crops(const Crop* crops, int s, bf16* x, float* t, float* kk, int nb, float tscale)
{
    const long per = WS_3D ? (long)s * s * s : (long)s * s;
    const long total = per * nb;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const int b = (int)(i / per);
        const Pix q = pix_of(i % per, s, s, s);
        const Crop c = crops[b];
        const long src = ((long)(c.z0 + q.z) * c.H + (c.y0 + q.y)) * c.W + (c.x0 + q.x);
        for (int ch = 0; ch < IN_PAD; ++ch)
            x[i * IN_PAD + ch] = ch < N_FEAT ? c.feat[src * N_FEAT + ch] : __float2bfloat16(0.f);
        t[i] = c.tgt[src] * tscale;
        for (int k = 0; k < NK; ++k) kk[NK * i + k] = c.kk[NK * src + k];
    }
}

// Sum of squares of n floats into *out (float32 atomics of block sums).
__global__ void k_sumsq(const float* v, long n, float* out)
{
    __shared__ float s[256];
    float a = 0.f;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) a += v[i] * v[i];
    s[threadIdx.x] = a;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(out, s[0]);
}

// ----------------------------------------------------------------------------- network

struct Conv {
    int cin, cout;
    float *w = nullptr, *b = nullptr, *gw = nullptr, *gb = nullptr, *mw = nullptr, *vw = nullptr, *mb = nullptr,
          *vb = nullptr;
    bf16 *w16 = nullptr, *wt16 = nullptr;
    bf16 *wpk16 = nullptr, *wtpk16 = nullptr;  // w16, wt16 in the MMA's shared-memory layout (k_pack_weights)
};

struct Pair {
    bf16* feat = nullptr;
    float* tgt = nullptr;
    float* kk = nullptr;  // (Kx, Ky[, Kz]) per cell
    int D = 1, H = 0, W = 0;
};

struct Net {
    int levels = 0, base = 0, device = 0;
    std::vector<int> ch;
    std::vector<Conv> conv;  // enc0a, enc0b, ..., enc(L-1)b, dec(L-2)a, dec(L-2)b, ..., dec0a, dec0b
    float *hw = nullptr, *hb = nullptr, *ghw = nullptr, *ghb = nullptr, *mh = nullptr, *vh = nullptr;  // head: C0 + 1
    long step = 0;
    int use_ref = 0;  // 1: CUDA-core convolutions
    int no_tma = 0;   // 1: the tensor-core convolutions without the TMA kernel
    cudaStream_t stream = nullptr;
    int* d_err = nullptr;
    float* d_sums = nullptr;
    double* d_scale = nullptr;
    double* d_partial = nullptr;
    float* d_img = nullptr;  // per-image residual sums of the training loss [2 * 256]
    double* r0buf = nullptr;  // the chunk's r0, [nz][ny][nx]
    long r0cap = 0;
    double* ubuf = nullptr;  // a pitched u-sized buffer for the smoothing sweeps
    long ucap = 0;
    // Workspace for n images of [D x] H x W; the training buffers (gradients, targets,
    // coefficients, loss) only when wtrain is set.
    int wn = 0, wD = 0, wH = 0, wW = 0;
    bool wtrain = false;
    std::vector<void*> wsbuf;
    bf16* x0 = nullptr;
    std::vector<bf16*> A, cat, P, DA, DB, gcat;
    bf16* bottom = nullptr;
    bf16 *G[3] = {nullptr, nullptr, nullptr};
    float *y = nullptr, *target = nullptr;
    float *kk = nullptr, *dbuf = nullptr, *ebuf = nullptr, *gy = nullptr;  // residual loss
    std::vector<Pair> pairs;
    Crop* d_crops = nullptr;
    int sms = 148;
    int smem_per_sm = 0, smem_reserved = 0, threads_per_sm = 0;
    float out_scale = 1.f;  // the network predicts du / max|u0| * out_scale (unit RMS on the pairs)
};

std::mutex g_mutex;
std::vector<std::unique_ptr<Net>>& nets()
{
    static std::vector<std::unique_ptr<Net>> v;
    return v;
}

Net* get_net(const int* id)
{
    auto& v = nets();
    if (!id || *id < 1 || (size_t)*id > v.size() || !v[*id - 1]) {
        set_status(TEA_ERR_BAD_ARGUMENT, "warm start: invalid network id %d", id ? *id : -1);
        return nullptr;
    }
    return v[*id - 1].get();
}

#define WS_CK(call)                                                                                       \
    do {                                                                                                  \
        cudaError_t e_ = (call);                                                                          \
        if (e_ != cudaSuccess) {                                                                          \
            set_status(TEA_ERR_CUDA, "warm start: %s failed: %s", #call, cudaGetErrorString(e_));       \
            return TEA_ERR_CUDA;                                                                          \
        }                                                                                                 \
    } while (0)

int grid_for(long work, int threads = 256)
{
    return (int)std::max<long>(1, std::min<long>((work + threads - 1) / threads, 148L * 16));
}

template <class T>
int dalloc(T** p, size_t count)
{
    WS_CK(cudaMalloc((void**)p, sizeof(T) * std::max<size_t>(count, 1)));
    WS_CK(cudaMemset(*p, 0, sizeof(T) * std::max<size_t>(count, 1)));
    // The clear runs on the legacy stream, which does not order with the library's
    // non-blocking streams: finish it before they use the memory.
    WS_CK(cudaDeviceSynchronize());
    return TEA_OK;
}

void free_workspace(Net* N)
{
    for (void* p : N->wsbuf) cudaFree(p);
    N->wsbuf.clear();
    N->A.clear();
    N->cat.clear();
    N->P.clear();
    N->DA.clear();
    N->DB.clear();
    N->gcat.clear();
    for (int k = 0; k < 3; ++k) N->G[k] = nullptr;
    N->target = N->kk = N->dbuf = N->ebuf = N->gy = nullptr;
    N->wn = N->wD = N->wH = N->wW = 0;
    N->wtrain = false;
}

// Depth of level l's images (1 in 2D).
inline int depth_at(const Net* N, int l) { return WS_3D ? N->wD >> l : 1; }

int ensure_workspace(Net* N, int n, int D, int H, int W, bool train)
{
    if (N->wn == n && N->wD == D && N->wH == H && N->wW == W && (N->wtrain || !train)) return TEA_OK;
    free_workspace(N);
    const int L = N->levels;
    auto take = [&](size_t bytes) -> void* {
        void* p = nullptr;
        if (cudaMalloc(&p, std::max<size_t>(bytes, 16)) != cudaSuccess) return nullptr;
        N->wsbuf.push_back(p);
        return p;
    };
    const long pix = (long)n * D * H * W;
    auto lv = [&](int l) { return pix >> (TEA_DIM * l); };
    bool ok = true;
    N->x0 = (bf16*)take(sizeof(bf16) * pix * IN_PAD);
    ok = ok && N->x0;
    N->A.resize(L);
    N->cat.resize(L);
    N->gcat.resize(L);
    N->P.resize(L);
    N->DA.resize(L);
    N->DB.resize(L);
    for (int l = 0; l < L; ++l) {
        N->A[l] = (bf16*)take(sizeof(bf16) * lv(l) * N->ch[l]);
        ok = ok && N->A[l];
        if (l < L - 1) {
            const int cc = N->ch[l + 1] + N->ch[l];
            N->cat[l] = (bf16*)take(sizeof(bf16) * lv(l) * cc);
            N->gcat[l] = (bf16*)take(sizeof(bf16) * lv(l) * cc);
            N->P[l] = (bf16*)take(sizeof(bf16) * lv(l + 1) * N->ch[l]);
            N->DA[l] = (bf16*)take(sizeof(bf16) * lv(l) * N->ch[l]);
            N->DB[l] = (bf16*)take(sizeof(bf16) * lv(l) * N->ch[l]);
            ok = ok && N->cat[l] && N->gcat[l] && N->P[l] && N->DA[l] && N->DB[l];
        }
    }
    N->bottom = (bf16*)take(sizeof(bf16) * lv(L - 1) * N->ch[L - 1]);
    N->y = (float*)take(sizeof(float) * pix);
    ok = ok && N->bottom && N->y;
    if (train) {
        for (int k = 0; k < 3; ++k) {
            N->G[k] = (bf16*)take(sizeof(bf16) * pix * N->ch[0]);
            ok = ok && N->G[k];
        }
        N->target = (float*)take(sizeof(float) * pix);
        N->kk = (float*)take(sizeof(float) * pix * NK);
        N->dbuf = (float*)take(sizeof(float) * pix);
        N->ebuf = (float*)take(sizeof(float) * pix);
        N->gy = (float*)take(sizeof(float) * pix);
        ok = ok && N->target && N->kk && N->dbuf && N->ebuf && N->gy;
    }
    if (!ok) {
        free_workspace(N);
        set_status(TEA_ERR_CUDA, "warm start: out of device memory for %d x %d x %d x %d", n, D, H, W);
        return TEA_ERR_CUDA;
    }
    N->wn = n;
    N->wD = D;
    N->wH = H;
    N->wW = W;
    N->wtrain = train;
    return TEA_OK;
}

// Blocks of a tensor-core kernel that fit on one SM at once: shared memory (with the
// per-block reservation), threads and tensor memory (512 columns per SM).  The occupancy API
// reports one block per SM for kernels that allocate tensor memory, whatever their size, so
// the count is formed here from the SM's resources.
int tc_blocks_per_sm(Net* N, int smem_bytes, int threads, int n_cols, int tmem_bufs = 1)
{
    if (N->smem_per_sm == 0) {
        cudaDeviceGetAttribute(&N->smem_per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, N->device);
        cudaDeviceGetAttribute(&N->smem_reserved, cudaDevAttrReservedSharedMemoryPerBlock, N->device);
        cudaDeviceGetAttribute(&N->threads_per_sm, cudaDevAttrMaxThreadsPerMultiProcessor, N->device);
    }
    const int by_smem = N->smem_per_sm / std::max(1, smem_bytes + N->smem_reserved);
    const int by_threads = N->threads_per_sm / threads;
    const int by_tmem = 512 / (tmem_bufs * tmem_cols(n_cols));
    return std::max(1, std::min(std::min(by_smem, by_threads), std::min(by_tmem, 32)));
}

// cuTensorMapEncodeTiled from the driver (looked up once; null when unavailable).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

// The tensor map of an input view for k_conv_tma: dims (channels of the view, W, H, D, n),
// boxes of 8 channels x 130 pixels x 1 x 1 x 1, zeros outside.  False when it cannot be made.
bool input_tensor_map(View x, int cin, int n, int D, int H, int W, CUtensorMap* map)
{
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc || (x.cs % 8) || (x.co % 8) || (cin % 8)) return false;
    const cuuint64_t dims[5] = {(cuuint64_t)cin, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)D, (cuuint64_t)n};
    const cuuint64_t px = (cuuint64_t)x.cs * sizeof(bf16);
    const cuuint64_t strides[4] = {px, px * W, px * W * H, px * W * H * D};
    const cuuint32_t box[5] = {8, 130, 1, 1, 1};
    const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, (void*)(x.p + x.co), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// y = conv(x) (3x3, or 3x3x3 in 3D) over n images of [D x] H x W; wpk is w packed by
// k_pack_weights (used by the TMA kernel).
void conv(Net* N, View x, View y, const bf16* w, const bf16* wpk, const float* bias, int relu, View mask, int n, int D,
          int H, int W, int cin, int cout)
{
    ConvArgs a;
    a.x = x.p;
    a.xcs = x.cs;
    a.xco = x.co;
    a.y = y.p;
    a.ycs = y.cs;
    a.yco = y.co;
    a.w = w;
    a.bias = bias;
    a.mask = mask.p;
    a.mcs = mask.cs;
    a.mco = mask.co;
    a.relu = relu;
    a.n = n;
    a.D = D;
    a.H = H;
    a.W = W;
    a.cin = cin;
    a.cout = cout;
    a.err = N->d_err;
    const long npix = (long)n * D * H * W;
    if (N->use_ref) {
        k_conv_ref<<<grid_for(npix * cout), 256, 0, N->stream>>>(a);
        return;
    }
    const long tiles = (npix + TC_M - 1) / TC_M;
    if (W % TC_M == 0 && wpk && !N->no_tma && conv_tma_smem_bytes(cin, cout, 2) <= 227 * 1024) {
        // Whole 128-pixel row tiles, every operand moved by TMA.
        CUtensorMap map;
        if (input_tensor_map(x, cin, n, D, H, W, &map)) {
            // As many stages (2..4) as leave room for two blocks per SM.
            const size_t stage = tma_stage_bytes(cin, cout);
            const int stages = (int)std::max<size_t>(2, std::min<size_t>(TMA_MAX_STAGES, (113 * 1024 - 1216) / stage));
            const int tbytes = (int)conv_tma_smem_bytes(cin, cout, stages);
            cudaFuncSetAttribute(k_conv_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, tbytes);
            const long grid =
                std::min<long>(tiles, (long)N->sms * tc_blocks_per_sm(N, tbytes, TMA_THREADS, pad16(cout), 2));
            k_conv_tma<<<(int)grid, TMA_THREADS, tbytes, N->stream>>>(a, wpk, stages, map);
            return;
        }
    }
    if (W % TC_M == 0 && conv_rows_smem_bytes(cin, cout) <= 227 * 1024) {
        // Rows of whole 128-pixel tiles: one staged row segment serves the three x-taps.
        const int rbytes = (int)conv_rows_smem_bytes(cin, cout);
        cudaFuncSetAttribute(k_conv_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, rbytes);
        const long grid = std::min<long>(tiles, (long)N->sms * tc_blocks_per_sm(N, rbytes, TC_THREADS, pad16(cout)));
        k_conv_rows<<<(int)grid, TC_THREADS, rbytes, N->stream>>>(a);
        return;
    }
    const int bytes = (int)conv_tc_smem_bytes(cin, cout);
    cudaFuncSetAttribute(k_conv_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    const long grid = std::min<long>(tiles, (long)N->sms * tc_blocks_per_sm(N, bytes, TC_THREADS, pad16(cout)));
    k_conv_tc<<<(int)grid, TC_THREADS, bytes, N->stream>>>(a);
}

void wgrad(Net* N, View x, View gy, Conv& L, int n, int D, int H, int W)
{
    const long npix = (long)n * D * H * W;
    // The tensor cores when the shapes fit their kernel (N = cin padded to 16, + 16 <= 256,
    // M = 128 >= cout, 16-byte channel groups), the CUDA cores otherwise and as the tests'
    // reference.
    const bool tc_fits = pad16(L.cin) + 16 <= 256 && L.cout <= 128 && L.cin % 8 == 0 && x.cs % 8 == 0 &&
                         x.co % 8 == 0 && gy.cs % 8 == 0 && gy.co % 8 == 0;
    if (!N->use_ref && tc_fits) {
        WgradArgs a;
        a.x = x.p;
        a.xcs = x.cs;
        a.xco = x.co;
        a.gy = gy.p;
        a.gcs = gy.cs;
        a.gco = gy.co;
        a.n = n;
        a.D = D;
        a.H = H;
        a.W = W;
        a.cin = L.cin;
        a.cout = L.cout;
        a.gw = L.gw;
        a.gb = L.gb;
        a.err = N->d_err;
        const int bytes = (int)wgrad_tc_smem_bytes(L.cin);
        cudaFuncSetAttribute(k_wgrad_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        const long resident = (long)N->sms * tc_blocks_per_sm(N, bytes, WT_THREADS, pad16(L.cin) + 16);
        const long slices = std::max<long>(1, std::min<long>((resident + TAPS - 1) / TAPS, (npix + WT_KP - 1) / WT_KP));
        k_wgrad_tc<<<dim3(TAPS, (unsigned)slices), WT_THREADS, bytes, N->stream>>>(a);
        return;
    }
    const int tiles = TAPS * ((L.cin + 31) / 32) * ((L.cout + 31) / 32);
    const int splits = (int)std::max<long>(1, std::min<long>((N->sms * 8 + tiles - 1) / tiles, (npix + 255) / 256));
    k_wgrad<<<dim3(tiles, splits), 256, 0, N->stream>>>(x.p, x.cs, x.co, gy.p, gy.cs, gy.co, n, D, H, W, L.cin,
                                                        L.cout, L.gw, L.gb);
}

View view(bf16* p, int cs, int co, int c)
{
    View v;
    v.p = p;
    v.cs = cs;
    v.co = co;
    v.c = c;
    return v;
}
const View kNoView = {nullptr, 0, 0, 0};

Conv& enc(Net* N, int l, int s) { return N->conv[2 * l + s]; }
Conv& dec(Net* N, int l, int s) { return N->conv[2 * N->levels + 2 * (N->levels - 2 - l) + s]; }

// Forward pass over the workspace's n images; x0 must hold the input.
void forward(Net* N)
{
    const int L = N->levels, n = N->wn;
    View h = view(N->x0, IN_PAD, 0, IN_PAD);
    for (int l = 0; l < L; ++l) {
        const int D = depth_at(N, l), H = N->wH >> l, W = N->wW >> l, C = N->ch[l];
        Conv& a = enc(N, l, 0);
        Conv& b = enc(N, l, 1);
        conv(N, h, view(N->A[l], C, 0, C), a.w16, a.wpk16, a.b, 1, kNoView, n, D, H, W, a.cin, C);
        const View out = l < L - 1 ? view(N->cat[l], N->ch[l + 1] + C, N->ch[l + 1], C) : view(N->bottom, C, 0, C);
        conv(N, view(N->A[l], C, 0, C), out, b.w16, b.wpk16, b.b, 1, kNoView, n, D, H, W, C, C);
        if (l < L - 1) {
            k_avgpool<<<grid_for((long)n * D * H * W / POOL), 256, 0, N->stream>>>(out, N->P[l], n, D, H, W);
            h = view(N->P[l], C, 0, C);
        }
    }
    for (int l = L - 2; l >= 0; --l) {
        const int D = depth_at(N, l), H = N->wH >> l, W = N->wW >> l, C = N->ch[l], Cu = N->ch[l + 1];
        const View hin = l == L - 2 ? view(N->bottom, Cu, 0, Cu) : view(N->DB[l + 1], Cu, 0, Cu);
        k_upsample<<<grid_for((long)n * D * H * W), 256, 0, N->stream>>>(hin, view(N->cat[l], Cu + C, 0, Cu), n,
                                                                              D, H, W);
        Conv& a = dec(N, l, 0);
        Conv& b = dec(N, l, 1);
        conv(N, view(N->cat[l], Cu + C, 0, Cu + C), view(N->DA[l], C, 0, C), a.w16, a.wpk16, a.b, 1, kNoView, n, D, H, W,
             Cu + C, C);
        conv(N, view(N->DA[l], C, 0, C), view(N->DB[l], C, 0, C), b.w16, b.wpk16, b.b, 1, kNoView, n, D, H, W, C, C);
    }
}

void head(Net* N, const float* target)
{
    const long npix = (long)N->wn * N->wD * N->wH * N->wW;
    const int C0 = N->ch[0];
    const int grid = grid_for(npix);
    if (C0 == 16)
        k_head<16><<<grid, 256, 0, N->stream>>>(N->DB[0], N->hw, N->hb, N->y, npix, target, N->d_sums, N->G[0],
                                                 N->ghw, N->ghb);
    else if (C0 == 24)
        k_head<24><<<grid, 256, 0, N->stream>>>(N->DB[0], N->hw, N->hb, N->y, npix, target, N->d_sums, N->G[0],
                                                 N->ghw, N->ghb);
    else if (C0 == 32)
        k_head<32><<<grid, 256, 0, N->stream>>>(N->DB[0], N->hw, N->hb, N->y, npix, target, N->d_sums, N->G[0],
                                                 N->ghw, N->ghb);
    else
        k_head<64><<<grid, 256, 0, N->stream>>>(N->DB[0], N->hw, N->hb, N->y, npix, target, N->d_sums, N->G[0],
                                                 N->ghw, N->ghb);
}

// Training loss: the energy norm (the norm CG minimises) of the smoothed guess's error
// relative to that of the plain start, per crop,
// L = (1/n) sum_b (M^k e_b).A(M^k e_b) / t_b.(A t_b), e_b = y_b - t_b (A the solver's operator
// with the crop's own Kx, Ky, no flux through the crop's edges; M^k the warm start's k damped
// Jacobi sweeps, which take care of the error's high frequencies and hence of most of the
// residual norm that decides whether a solve uses the guess); every timestep alike.  Writes dL/dh into G[0] and the head's gradients;
// d_img[2b], d_img[2b + 1] receive |A (y_b - t_b)|^2 and |A t_b|^2.
void residual_loss_backward(Net* N)
{
    const int n = N->wn, D = N->wD, H = N->wH, W = N->wW;
    const long npix = (long)n * D * H * W;
    const int grid = grid_for(npix);
    const dim3 g2(std::max(1, grid_for((long)D * H * W) / std::max(1, n / 8 + 1)), n);
    cudaMemsetAsync(N->d_img, 0, sizeof(float) * 2 * n, N->stream);
    // d = y - t, then WS_SMOOTH damped Jacobi sweeps of the error (ping-pong d <-> gy).
    k_res_loss<<<g2, 256, 0, N->stream>>>(N->y, N->target, N->kk, N->dbuf, N->ebuf, D, H, W, N->d_img, 0);
    float* a = N->dbuf;
    float* b = N->gy;
    for (int k = 0; k < WS_SMOOTH; ++k) {
        k_smooth_err<<<grid, 256, 0, N->stream>>>(a, nullptr, b, N->kk, n, D, H, W, 0);
        std::swap(a, b);
    }
    if (a != N->dbuf) cudaMemcpyAsync(N->dbuf, a, sizeof(float) * npix, cudaMemcpyDeviceToDevice, N->stream);
    // e = A M^k (y - t); sums; g = 2 A M^k (y - t) / (n t.A t), then back through the sweeps.
    k_res_loss<<<g2, 256, 0, N->stream>>>(N->y, N->target, N->kk, N->dbuf, N->ebuf, D, H, W, N->d_img, 1);
    k_res_grad<<<g2, 256, 0, N->stream>>>(N->ebuf, N->kk, N->d_img, N->gy, n, D, H, W);
    a = N->gy;
    b = N->dbuf;
    for (int k = 0; k < WS_SMOOTH; ++k) {
        k_dinv<<<grid, 256, 0, N->stream>>>(a, N->ebuf, N->kk, n, D, H, W);
        k_smooth_err<<<grid, 256, 0, N->stream>>>(a, N->ebuf, b, N->kk, n, D, H, W, 1);
        std::swap(a, b);
    }
    if (a != N->gy) cudaMemcpyAsync(N->gy, a, sizeof(float) * npix, cudaMemcpyDeviceToDevice, N->stream);
    const int C0 = N->ch[0];
    if (C0 == 16)
        k_head_bw<16><<<grid, 256, 0, N->stream>>>(N->DB[0], N->hw, N->gy, npix, N->G[0], N->ghw, N->ghb);
    else if (C0 == 24)
        k_head_bw<24><<<grid, 256, 0, N->stream>>>(N->DB[0], N->hw, N->gy, npix, N->G[0], N->ghw, N->ghb);
    else if (C0 == 32)
        k_head_bw<32><<<grid, 256, 0, N->stream>>>(N->DB[0], N->hw, N->gy, npix, N->G[0], N->ghw, N->ghb);
    else
        k_head_bw<64><<<grid, 256, 0, N->stream>>>(N->DB[0], N->hw, N->gy, npix, N->G[0], N->ghw, N->ghb);
}

// Backward pass after forward() and the head's backward: accumulates every parameter gradient.
void backward(Net* N)
{
    const int L = N->levels, n = N->wn;
    bf16* gcur = N->G[0];  // gradient w.r.t. the pre-activation of dec0b (from the head)
    bf16* gnext = N->G[1];
    bf16* gtmp = N->G[2];
    for (int l = 0; l <= L - 2; ++l) {
        const int D = depth_at(N, l), H = N->wH >> l, W = N->wW >> l, C = N->ch[l], Cu = N->ch[l + 1];
        Conv& a = dec(N, l, 0);
        Conv& b = dec(N, l, 1);
        wgrad(N, view(N->DA[l], C, 0, C), view(gcur, C, 0, C), b, n, D, H, W);
        conv(N, view(gcur, C, 0, C), view(gnext, C, 0, C), b.wt16, b.wtpk16, nullptr, 0, view(N->DA[l], C, 0, C), n, D, H, W,
             C, C);
        wgrad(N, view(N->cat[l], Cu + C, 0, Cu + C), view(gnext, C, 0, C), a, n, D, H, W);
        conv(N, view(gnext, C, 0, C), view(N->gcat[l], Cu + C, 0, Cu + C), a.wt16, a.wtpk16, nullptr, 0,
             view(N->cat[l], Cu + C, 0, Cu + C), n, D, H, W, C, Cu + C);
        k_upsample_bw<<<grid_for((long)n * D * H * W / POOL), 256, 0, N->stream>>>(
            view(N->gcat[l], Cu + C, 0, Cu), gcur, n, D, H, W);
    }
    // gcur: gradient w.r.t. the pre-activation of enc(L-1)b.
    for (int l = L - 1; l >= 0; --l) {
        const int D = depth_at(N, l), H = N->wH >> l, W = N->wW >> l, C = N->ch[l];
        Conv& a = enc(N, l, 0);
        Conv& b = enc(N, l, 1);
        if (l < L - 1) {
            // gcur holds the gradient w.r.t. the pooled tensor P[l] (coarse); add the skip's.
            const int Cu = N->ch[l + 1];
            k_avgpool_bw<<<grid_for((long)n * D * H * W), 256, 0, N->stream>>>(
                gcur, view(N->cat[l], Cu + C, Cu, C), view(N->gcat[l], Cu + C, Cu, C), gtmp, n, D, H, W);
            std::swap(gcur, gtmp);
        }
        wgrad(N, view(N->A[l], C, 0, C), view(gcur, C, 0, C), b, n, D, H, W);
        conv(N, view(gcur, C, 0, C), view(gnext, C, 0, C), b.wt16, b.wtpk16, nullptr, 0, view(N->A[l], C, 0, C), n, D, H, W, C,
             C);
        const View xin = l == 0 ? view(N->x0, IN_PAD, 0, IN_PAD) : view(N->P[l - 1], N->ch[l - 1], 0, N->ch[l - 1]);
        wgrad(N, xin, view(gnext, C, 0, C), a, n, D, H, W);
        if (l > 0) {
            const int Cp = N->ch[l - 1];
            conv(N, view(gnext, C, 0, C), view(gcur, Cp, 0, Cp), a.wt16, a.wtpk16, nullptr, 0, kNoView, n, D, H, W, C, Cp);
        }
    }
}

void refresh_bf16(Net* N)
{
    for (Conv& c : N->conv) {
        k_weights_bf16<<<grid_for((long)c.cout * TAPS * c.cin), 256, 0, N->stream>>>(c.w, c.w16, c.wt16, c.cout,
                                                                                      c.cin);
        k_pack_weights<<<grid_for((long)TAPS * pad16(c.cout) * pad16(c.cin)), 256, 0, N->stream>>>(c.w16, c.wpk16,
                                                                                                 c.cout, c.cin);
        k_pack_weights<<<grid_for((long)TAPS * pad16(c.cout) * pad16(c.cin)), 256, 0, N->stream>>>(c.wt16, c.wtpk16,
                                                                                                 c.cin, c.cout);
    }
}

void adam_step(Net* N, float lr)
{
    N->step += 1;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float c1 = 1.f - powf(b1, (float)N->step), c2 = 1.f - powf(b2, (float)N->step);
    for (Conv& c : N->conv) {
        const long nw = (long)c.cout * TAPS * c.cin;
        k_adam<<<grid_for(nw), 256, 0, N->stream>>>(c.w, c.gw, c.mw, c.vw, nw, lr, b1, b2, eps, c1, c2);
        k_adam<<<grid_for(c.cout), 256, 0, N->stream>>>(c.b, c.gb, c.mb, c.vb, c.cout, lr, b1, b2, eps, c1, c2);
    }
    const int nh = N->ch[0] + 1;  // head weights and bias are contiguous
    k_adam<<<1, 256, 0, N->stream>>>(N->hw, N->ghw, N->mh, N->vh, nh, lr, b1, b2, eps, c1, c2);
    refresh_bf16(N);
}

int cin_of_oracle(const Net* N, int k) { return k == 0 ? N_FEAT : N->conv[k].cin; }

// Parameters in the oracle's order (oracle/warmstart_oracle.py layer_shapes): per layer
// w[co][TAPS][cin] (cin of the first layer: the real features) then b; head w, head b.
long param_count(const Net* N)
{
    long n = 0;
    for (size_t k = 0; k < N->conv.size(); ++k)
        n += (long)N->conv[k].cout * TAPS * cin_of_oracle(N, (int)k) + N->conv[k].cout;
    return n + N->ch[0] + 1;
}

// Copy between host oracle-order arrays and the device (w: master weights, or gradients).
int transfer_params(Net* N, float* host, bool to_device, bool grads)
{
    long off = 0;
    std::vector<float> buf;
    for (size_t k = 0; k < N->conv.size(); ++k) {
        Conv& c = N->conv[k];
        const int ci_o = cin_of_oracle(N, (int)k);
        buf.assign((size_t)c.cout * TAPS * c.cin, 0.f);
        float* dw = grads ? c.gw : c.w;
        float* db = grads ? c.gb : c.b;
        if (to_device) {
            for (int co = 0; co < c.cout; ++co)
                for (int t = 0; t < TAPS; ++t)
                    for (int ci = 0; ci < ci_o; ++ci)
                        buf[((size_t)co * TAPS + t) * c.cin + ci] = host[off + ((long)co * TAPS + t) * ci_o + ci];
            WS_CK(copy_on(N->stream, dw, buf.data(), sizeof(float) * buf.size(), cudaMemcpyHostToDevice));
            WS_CK(copy_on(N->stream, db, host + off + (long)c.cout * TAPS * ci_o, sizeof(float) * c.cout,
                          cudaMemcpyHostToDevice));
        } else {
            WS_CK(copy_on(N->stream, buf.data(), dw, sizeof(float) * buf.size(), cudaMemcpyDeviceToHost));
            for (int co = 0; co < c.cout; ++co)
                for (int t = 0; t < TAPS; ++t)
                    for (int ci = 0; ci < ci_o; ++ci)
                        host[off + ((long)co * TAPS + t) * ci_o + ci] = buf[((size_t)co * TAPS + t) * c.cin + ci];
            WS_CK(copy_on(N->stream, host + off + (long)c.cout * TAPS * ci_o, db, sizeof(float) * c.cout,
                          cudaMemcpyDeviceToHost));
        }
        off += (long)c.cout * TAPS * ci_o + c.cout;
    }
    const int nh = N->ch[0] + 1;
    float* dh = grads ? N->ghw : N->hw;
    if (to_device)
        WS_CK(copy_on(N->stream, dh, host + off, sizeof(float) * nh, cudaMemcpyHostToDevice));
    else
        WS_CK(copy_on(N->stream, host + off, dh, sizeof(float) * nh, cudaMemcpyDeviceToHost));
    if (to_device && !grads) refresh_bf16(N);
    return TEA_OK;
}

int check_err(Net* N, const char* what)
{
    WS_CK(cudaStreamSynchronize(N->stream));
    int e = 0;
    WS_CK(copy_on(N->stream, &e, N->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) {
        set_status(TEA_ERR_CUDA, "warm start: %s: a tensor-core wait timed out", what);
        int z = 0;
        copy_on(N->stream, N->d_err, &z, sizeof(int), cudaMemcpyHostToDevice);
        return TEA_ERR_CUDA;
    }
    return TEA_OK;
}

// Features of the chunk's step into x0 (and the scale max |r0| into d_scale), on `stream`.
int chunk_features(Net* N, Chunk* c, cudaStream_t stream)
{
    const Geom& g = c->g;
    const long pix = inner_cells(g);
    if (N->r0cap < pix) {
        if (N->r0buf) cudaFree(N->r0buf);
        N->r0buf = nullptr;
        N->r0cap = 0;
        if (dalloc(&N->r0buf, pix)) return TEA_ERR_CUDA;
        N->r0cap = pix;
    }
    const int blocks = 512;
    k_r0<<<grid_for(pix), 256, 0, stream>>>(g, c->f.u0, c->f.kx, c->f.ky, c->f.kz, N->r0buf);
    k_absmax<<<blocks, 256, 0, stream>>>(N->r0buf, pix, N->d_partial);
    k_absmax_final<<<1, 256, 0, stream>>>(N->d_partial, blocks, N->d_scale);
    k_features<<<grid_for(pix), 256, 0, stream>>>(g, N->r0buf, c->f.density, c->f.kx, c->f.ky, c->f.kz, N->d_scale,
                                                  N->x0);
    return TEA_OK;
}

// Whether the chunk's inner extents divide by 2^(levels - 1) (every level pools by 2).
bool chunk_fits(const Net* N, const Geom& g)
{
    const int div = 1 << (N->levels - 1);
    return g.nx % div == 0 && g.ny % div == 0 && (!WS_3D || g.nz % div == 0);
}

// The chunk's images: one image of [nz x] ny x nx.
int chunk_depth(const Geom& g) { return WS_3D ? g.nz : 1; }

}  // namespace ws

// ----------------------------------------------------------------------------- solve hook

// Called by ext_tea_leaf_solve_ after the CG set-up (u = u0, r, p, rro): predicts
// du, and keeps u = u0 + du when its initial residual is smaller.  Returns 1 when the
// guess was kept (the caller then re-initialises r, p and rro from it), 0 otherwise.
int ws_predict_into(Chunk* c, double* u_out)
{
    using namespace ws;
    Net* N = static_cast<Net*>(c->ws);
    if (!N) return 0;
    const Geom& g = c->g;
    if (!chunk_fits(N, g)) return 0;
    if (ensure_workspace(N, 1, chunk_depth(g), g.ny, g.nx, false) != TEA_OK) return 0;
    cudaStream_t saved = N->stream;
    N->stream = c->stream;
    if (chunk_features(N, c, c->stream) != TEA_OK) {
        N->stream = saved;
        return 0;
    }
    forward(N);
    head(N, nullptr);
    // Guess into u, then WS_SMOOTH (even) damped Jacobi sweeps ping-ponged through a second
    // pitched buffer, ending in u; only inner cells are written.
    if (N->ucap < (long)c->field_elems) {
        if (N->ubuf) cudaFree(N->ubuf);
        N->ubuf = nullptr;
        N->ucap = 0;
        if (dalloc(&N->ubuf, c->field_elems)) {
            N->stream = saved;
            return 0;
        }
        N->ucap = (long)c->field_elems;
    }
    static_assert(WS_SMOOTH % 2 == 0, "the sweeps must end in u");
    k_apply_guess<<<grid_for(inner_cells(g)), 256, 0, c->stream>>>(g, N->y, c->f.u0, N->d_scale,
                                                                    1.0 / (double)N->out_scale, u_out);
    double* src = u_out;
    double* dst = N->ubuf + kLeadPad;
    for (int k = 0; k < WS_SMOOTH; ++k) {
        k_ws_smooth<<<grid_for(inner_cells(g)), 256, 0, c->stream>>>(g, src, c->f.u0, c->f.kx, c->f.ky, c->f.kz,
                                                                     dst);
        std::swap(src, dst);
    }
    N->stream = saved;
    return 1;
}

}  // namespace tea

using namespace tea;
using namespace tea::ws;

TEA_EXPORT int tea_ws_create_capped_(const int* levels, const int* base, const int* max_channels, const int* seed,
                                     int* net)
{
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!levels || !base || !max_channels || !net || *levels < 2 || *levels > 5 ||
        (*base != 16 && *base != 24 && *base != 32 && *base != 64) || *max_channels < 0 || *max_channels % 8) {
        set_status(TEA_ERR_BAD_ARGUMENT,
                   "tea_ws_create_: levels must be 2..5, base 16, 24, 32 or 64, max_channels a multiple of 8");
        return TEA_ERR_BAD_ARGUMENT;
    }
    // Channels double per level, up to max_channels (0: no limit).  Every layer must fit the
    // tensor-core kernels: N = Cout padded to 16 at most 256, and two stages of the operand
    // tiles in shared memory.
    std::vector<int> ch;
    for (int l = 0; l < *levels; ++l)
        ch.push_back(*max_channels > 0 ? std::min(*base << l, std::max(*max_channels, *base)) : *base << l);
    const int deepest_cat = ch.back() + ch[*levels - 2];
    if (pad16(ch.back()) > 256 || conv_tc_smem_bytes(deepest_cat, ch[*levels - 2]) > 227 * 1024 ||
        conv_tc_smem_bytes(ch.back(), ch.back()) > 227 * 1024) {
        set_status(TEA_ERR_BAD_ARGUMENT, "tea_ws_create_: too many channels for one tensor-core tile");
        return TEA_ERR_BAD_ARGUMENT;
    }
    auto N = std::make_unique<Net>();
    N->levels = *levels;
    N->base = *base;
    N->ch = ch;
    WS_CK(cudaGetDevice(&N->device));
    WS_CK(cudaDeviceGetAttribute(&N->sms, cudaDevAttrMultiProcessorCount, N->device));
    WS_CK(cudaStreamCreateWithFlags(&N->stream, cudaStreamNonBlocking));
    int prev = IN_PAD;
    for (int l = 0; l < N->levels; ++l) {
        N->conv.push_back({prev, N->ch[l]});
        N->conv.push_back({N->ch[l], N->ch[l]});
        prev = N->ch[l];
    }
    for (int l = N->levels - 2; l >= 0; --l) {
        N->conv.push_back({N->ch[l + 1] + N->ch[l], N->ch[l]});
        N->conv.push_back({N->ch[l], N->ch[l]});
    }
    // He initialisation (the first layer over its real inputs), small biases; seeded.
    std::mt19937_64 rng((unsigned long long)(seed ? *seed : 0));
    std::normal_distribution<float> nd(0.f, 1.f);
    for (size_t k = 0; k < N->conv.size(); ++k) {
        Conv& c = N->conv[k];
        const long nw = (long)c.cout * TAPS * c.cin;
        for (float** p : {&c.w, &c.gw, &c.mw, &c.vw})
            if (dalloc(p, nw)) return TEA_ERR_CUDA;
        for (float** p : {&c.b, &c.gb, &c.mb, &c.vb})
            if (dalloc(p, c.cout)) return TEA_ERR_CUDA;
        if (dalloc(&c.w16, nw) || dalloc(&c.wt16, nw)) return TEA_ERR_CUDA;
        const long npk = (long)TAPS * pad16(c.cout) * pad16(c.cin);
        if (dalloc(&c.wpk16, npk) || dalloc(&c.wtpk16, npk)) return TEA_ERR_CUDA;
        const int ci_real = k == 0 ? N_FEAT : c.cin;
        const float sd = sqrtf(2.f / ((float)TAPS * ci_real));
        std::vector<float> w(nw, 0.f), b(c.cout);
        for (int co = 0; co < c.cout; ++co)
            for (int t = 0; t < TAPS; ++t)
                for (int ci = 0; ci < ci_real; ++ci) w[((long)co * TAPS + t) * c.cin + ci] = sd * nd(rng);
        for (auto& v : b) v = 0.01f * nd(rng);
        WS_CK(copy_on(N->stream, c.w, w.data(), sizeof(float) * nw, cudaMemcpyHostToDevice));
        WS_CK(copy_on(N->stream, c.b, b.data(), sizeof(float) * c.cout, cudaMemcpyHostToDevice));
    }
    const int nh = N->ch[0] + 1;
    for (float** p : {&N->hw, &N->ghw, &N->mh, &N->vh})
        if (dalloc(p, nh)) return TEA_ERR_CUDA;
    N->hb = N->hw + N->ch[0];
    N->ghb = N->ghw + N->ch[0];
    // The head starts at zero: the untrained guess is du = 0, the plain start itself.
    if (dalloc(&N->d_err, 1) || dalloc(&N->d_sums, 4) || dalloc(&N->d_scale, 1) || dalloc(&N->d_partial, 512) ||
        dalloc(&N->d_crops, 256) || dalloc(&N->d_img, 512))
        return TEA_ERR_CUDA;
    refresh_bf16(N.get());
    WS_CK(cudaStreamSynchronize(N->stream));
    nets().push_back(std::move(N));
    *net = (int)nets().size();
    return TEA_OK;
}

TEA_EXPORT int tea_ws_create_(const int* levels, const int* base, const int* seed, int* net)
{
    const int unlimited = 0;
    return tea_ws_create_capped_(levels, base, &unlimited, seed, net);
}

TEA_EXPORT int tea_ws_destroy_(const int* net)
{
    std::lock_guard<std::mutex> lock(g_mutex);
    Net* N = get_net(net);
    if (!N) return TEA_ERR_BAD_ARGUMENT;
    cudaStreamSynchronize(N->stream);
    free_workspace(N);
    for (Conv& c : N->conv)
        for (void* p : {(void*)c.w, (void*)c.b, (void*)c.gw, (void*)c.gb, (void*)c.mw, (void*)c.vw, (void*)c.mb,
                        (void*)c.vb, (void*)c.w16, (void*)c.wt16, (void*)c.wpk16, (void*)c.wtpk16})
            cudaFree(p);
    for (void* p : {(void*)N->hw, (void*)N->ghw, (void*)N->mh, (void*)N->vh, (void*)N->d_err, (void*)N->d_sums,
                    (void*)N->d_scale, (void*)N->d_partial, (void*)N->d_crops, (void*)N->d_img, (void*)N->r0buf,
                    (void*)N->ubuf})
        cudaFree(p);
    for (Pair& p : N->pairs) {
        cudaFree(p.feat);
        cudaFree(p.tgt);
        cudaFree(p.kk);
    }
    cudaStreamDestroy(N->stream);
    nets()[*net - 1].reset();
    return TEA_OK;
}

TEA_EXPORT int tea_ws_set_conv_(const int* net, const int* reference)
{
    Net* N = get_net(net);
    if (!N) return TEA_ERR_BAD_ARGUMENT;
    N->use_ref = *reference == 1 ? 1 : 0;
    N->no_tma = *reference == 2 ? 1 : 0;
    return TEA_OK;
}

TEA_EXPORT int tea_ws_param_count_(const int* net, long long* count)
{
    Net* N = get_net(net);
    if (!N) return TEA_ERR_BAD_ARGUMENT;
    *count = param_count(N);
    return TEA_OK;
}

TEA_EXPORT int tea_ws_get_params_(const int* net, float* params)
{
    Net* N = get_net(net);
    if (!N) return TEA_ERR_BAD_ARGUMENT;
    return transfer_params(N, params, false, false);
}

TEA_EXPORT int tea_ws_set_params_(const int* net, const float* params)
{
    Net* N = get_net(net);
    if (!N) return TEA_ERR_BAD_ARGUMENT;
    const int rc = transfer_params(N, const_cast<float*>(params), true, false);
    if (rc == TEA_OK) WS_CK(cudaStreamSynchronize(N->stream));
    return rc;
}

// Forward (and, with a target, backward) over n host images of the features
// [n][D][H][W][N_FEAT] (D = 1 in the 2D library); writes the prediction [n][D][H][W], the
// loss and the parameter gradients (oracle order).  The loss is the mean squared error, or
// with kxy ([n][D][H][W][NK] face coefficients) the training's residual loss.
TEA_EXPORT int tea_ws_eval_volume_(const int* net, const float* x, const float* target, const float* kxy,
                                   const int* n, const int* D, const int* H, const int* W, float* y, double* loss,
                                   float* grads)
{
    Net* N = get_net(net);
    if (!N || !x || !y || !n || !D || !H || !W || *n < 1 || *D < 1 || *H < 2 || *W < 2 || (!WS_3D && *D != 1))
        return TEA_ERR_BAD_ARGUMENT;
    const int div = 1 << (N->levels - 1);
    if (*H % div || *W % div || (WS_3D && *D % div)) {
        set_status(TEA_ERR_BAD_ARGUMENT, "warm start: image sides must be multiples of %d", div);
        return TEA_ERR_BAD_ARGUMENT;
    }
    int rc = ensure_workspace(N, *n, *D, *H, *W, target != nullptr);
    if (rc) return rc;
    const long pix = (long)*n * *D * *H * *W;
    std::vector<bf16> hx(pix * IN_PAD, __float2bfloat16(0.f));
    for (long p = 0; p < pix; ++p)
        for (int c = 0; c < N_FEAT; ++c) hx[p * IN_PAD + c] = __float2bfloat16(x[p * N_FEAT + c]);
    WS_CK(cudaMemcpyAsync(N->x0, hx.data(), sizeof(bf16) * hx.size(), cudaMemcpyHostToDevice, N->stream));
    if (target) {
        WS_CK(cudaMemcpyAsync(N->target, target, sizeof(float) * pix, cudaMemcpyHostToDevice, N->stream));
        WS_CK(cudaMemsetAsync(N->d_sums, 0, sizeof(float) * 4, N->stream));
        for (Conv& c : N->conv) {
            WS_CK(cudaMemsetAsync(c.gw, 0, sizeof(float) * c.cout * TAPS * c.cin, N->stream));
            WS_CK(cudaMemsetAsync(c.gb, 0, sizeof(float) * c.cout, N->stream));
        }
        WS_CK(cudaMemsetAsync(N->ghw, 0, sizeof(float) * (N->ch[0] + 1), N->stream));
    }
    forward(N);
    if (target && kxy) {
        WS_CK(cudaMemcpyAsync(N->kk, kxy, sizeof(float) * pix * NK, cudaMemcpyHostToDevice, N->stream));
        head(N, nullptr);
        residual_loss_backward(N);
    } else {
        head(N, target ? N->target : nullptr);
    }
    if (target) backward(N);
    if ((rc = check_err(N, "eval"))) return rc;
    WS_CK(copy_on(N->stream, y, N->y, sizeof(float) * pix, cudaMemcpyDeviceToHost));
    if (target) {
        if (kxy) {
            std::vector<float> v(2 * (size_t)*n);
            WS_CK(copy_on(N->stream, v.data(), N->d_img, sizeof(float) * v.size(), cudaMemcpyDeviceToHost));
            double r = 0.0;
            for (int b = 0; b < *n; ++b) r += v[2 * b + 1] > 0.f ? (double)v[2 * b] / v[2 * b + 1] : 0.0;
            if (loss) *loss = r / *n;
        } else {
            float s = 0.f;
            WS_CK(copy_on(N->stream, &s, N->d_sums, sizeof(float), cudaMemcpyDeviceToHost));
            if (loss) *loss = (double)s / (double)pix;
        }
        if (grads && (rc = transfer_params(N, grads, false, true))) return rc;
    }
    return TEA_OK;
}

// tea_ws_eval_volume_ over images of depth 1: [n][H][W][N_FEAT] features.
TEA_EXPORT int tea_ws_eval_host_(const int* net, const float* x, const float* target, const float* kxy,
                                 const int* n, const int* H, const int* W, float* y, double* loss, float* grads)
{
    const int one = 1;
    return tea_ws_eval_volume_(net, x, target, kxy, n, &one, H, W, y, loss, grads);
}

// Records a training pair from the chunk's last solve: the step's features and
// (u - u0) / scale.  Call after ext_tea_leaf_solve_ (u holds the solution, u0 the step's
// right-hand side).
TEA_EXPORT int tea_ws_record_(const int* net, const int* chunk)
{
    Net* N = get_net(net);
    Chunk* c = get_chunk(chunk);
    if (!N || !c) return TEA_ERR_BAD_ARGUMENT;
    const Geom& g = c->g;
    int rc = ensure_workspace(N, 1, chunk_depth(g), g.ny, g.nx, false);
    if (rc) return rc;
    Pair p;
    p.D = chunk_depth(g);
    p.H = g.ny;
    p.W = g.nx;
    const long pix = inner_cells(g);
    if (dalloc(&p.feat, pix * N_FEAT) || dalloc(&p.tgt, pix) || dalloc(&p.kk, pix * NK)) return TEA_ERR_CUDA;
    WS_CK(cudaStreamSynchronize(c->stream));
    if ((rc = chunk_features(N, c, N->stream))) return rc;
    k_record<<<grid_for(pix), 256, 0, N->stream>>>(g, N->x0, c->f.u, c->f.u0, c->f.kx, c->f.ky, c->f.kz, N->d_scale,
                                                   p.feat, p.tgt, p.kk);
    WS_CK(cudaStreamSynchronize(N->stream));
    N->pairs.push_back(p);
    return TEA_OK;
}

TEA_EXPORT int tea_ws_pairs_(const int* net, int* count)
{
    Net* N = get_net(net);
    if (!N) return TEA_ERR_BAD_ARGUMENT;
    *count = (int)N->pairs.size();
    return TEA_OK;
}

// `steps` Adam steps on batches of `batch` random crop x crop (x crop in 3D) windows of the
// recorded pairs.
TEA_EXPORT int tea_ws_train_(const int* net, const int* steps, const int* batch, const int* crop, const double* lr,
                             const int* seed, double* loss_first, double* loss_last, double* ms_per_step)
{
    Net* N = get_net(net);
    if (!N) return TEA_ERR_BAD_ARGUMENT;
    const int div = 1 << (N->levels - 1);
    if (N->pairs.empty() || *steps < 1 || *batch < 1 || *batch > 256 || *crop < div || *crop % div) {
        set_status(TEA_ERR_BAD_ARGUMENT, "tea_ws_train_: needs recorded pairs, 1..256 crops a multiple of %d", div);
        return TEA_ERR_BAD_ARGUMENT;
    }
    for (const Pair& p : N->pairs)
        if (p.H < *crop || p.W < *crop || (WS_3D && p.D < *crop)) {
            set_status(TEA_ERR_BAD_ARGUMENT, "tea_ws_train_: crop larger than a recorded pair");
            return TEA_ERR_BAD_ARGUMENT;
        }
    const int cd = WS_3D ? *crop : 1;  // crop depth
    int rc = ensure_workspace(N, *batch, cd, *crop, *crop, true);
    if (rc) return rc;
    std::mt19937_64 rng((unsigned long long)(seed ? *seed : 0));
    std::vector<Crop> crops(*batch);
    const long pix = (long)*batch * cd * *crop * *crop;
    if (N->step == 0) {
        // Targets normalised to unit RMS over the recorded pairs (fixed at the first training).
        WS_CK(cudaMemsetAsync(N->d_sums + 1, 0, sizeof(float), N->stream));
        long total = 0;
        for (const Pair& p : N->pairs) {
            const long n = (long)p.D * p.H * p.W;
            k_sumsq<<<grid_for(n), 256, 0, N->stream>>>(p.tgt, n, N->d_sums + 1);
            total += n;
        }
        float ss = 0.f;
        WS_CK(cudaMemcpyAsync(&ss, N->d_sums + 1, sizeof(float), cudaMemcpyDeviceToHost, N->stream));
        WS_CK(cudaStreamSynchronize(N->stream));
        const double rms = std::sqrt((double)ss / (double)std::max<long>(total, 1));
        N->out_scale = rms > 0.0 ? (float)(1.0 / rms) : 1.f;
    }
    const int win = std::max(1, std::min(10, *steps / 2));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double first = 0.0, last = 0.0;
    for (int s = 0; s < *steps; ++s) {
        for (int b = 0; b < *batch; ++b) {
            const Pair& p = N->pairs[rng() % N->pairs.size()];
            crops[b].feat = p.feat;
            crops[b].tgt = p.tgt;
            crops[b].kk = p.kk;
            crops[b].H = p.H;
            crops[b].W = p.W;
            crops[b].y0 = (int)(rng() % (unsigned long long)(p.H - *crop + 1));
            crops[b].x0 = (int)(rng() % (unsigned long long)(p.W - *crop + 1));
            crops[b].z0 = WS_3D ? (int)(rng() % (unsigned long long)(p.D - *crop + 1)) : 0;
        }
        WS_CK(cudaMemcpyAsync(N->d_crops, crops.data(), sizeof(Crop) * crops.size(), cudaMemcpyHostToDevice,
                              N->stream));
        if (s == 1) cudaEventRecord(e0, N->stream);
        k_crops<<<grid_for(pix), 256, 0, N->stream>>>(N->d_crops, *crop, N->x0, N->target, N->kk, *batch,
                                                       N->out_scale);
        forward(N);
        head(N, nullptr);
        residual_loss_backward(N);
        backward(N);
        adam_step(N, (float)*lr);
        // The reported losses average the first and the last `win` steps.
        if (s < win || s >= *steps - win) {
            std::vector<float> v(2 * (size_t)*batch);
            WS_CK(cudaMemcpyAsync(v.data(), N->d_img, sizeof(float) * v.size(), cudaMemcpyDeviceToHost, N->stream));
            WS_CK(cudaStreamSynchronize(N->stream));
            float dmax = 0.f;
            for (int b = 0; b < *batch; ++b) dmax = std::max(dmax, v[2 * b + 1]);
            double r = 0.0;
            for (int b = 0; b < *batch; ++b) r += (double)v[2 * b] / std::max(std::max(v[2 * b + 1], 1e-3f * dmax), 1e-30f);
            r /= *batch;
            if (s < win) first += r / win;
            if (s >= *steps - win) last += r / win;
        }
    }
    cudaEventRecord(e1, N->stream);
    if ((rc = check_err(N, "train"))) return rc;
    float ms = 0.f;
    if (*steps > 1) cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (loss_first) *loss_first = first;
    if (loss_last) *loss_last = last;
    if (ms_per_step) *ms_per_step = *steps > 1 ? ms / (*steps - 1) : 0.0;
    return TEA_OK;
}

// Attaches a network to a chunk (net 0 detaches): the chunk's whole-solve calls then start
// from the network's prediction when it has the smaller initial residual.
TEA_EXPORT int tea_ws_attach_(const int* chunk, const int* net)
{
    Chunk* c = get_chunk(chunk);
    if (!c) return TEA_ERR_BAD_ARGUMENT;
    if (!net || *net == 0) {
        c->ws = nullptr;
        return TEA_OK;
    }
    Net* N = get_net(net);
    if (!N) return TEA_ERR_BAD_ARGUMENT;
    c->ws = N;
    c->ws_reject_streak = 0;
    c->ws_skip = 0;
    return TEA_OK;
}

// Prediction on the chunk's current step (features from u0, density, Kx, Ky[, Kz]) into a
// host array [nz][ny][nx] of du, and the milliseconds the network took on the device.
TEA_EXPORT int tea_ws_predict_(const int* net, const int* chunk, double* du, double* ms)
{
    Net* N = get_net(net);
    Chunk* c = get_chunk(chunk);
    if (!N || !c) return TEA_ERR_BAD_ARGUMENT;
    void* saved = c->ws;  // (du below is in units of u: the output normalisation is undone)
    c->ws = N;
    const Geom& g = c->g;
    double* tmp = nullptr;
    const long pix = inner_cells(g);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    WS_CK(cudaMalloc(&tmp, sizeof(double) * c->field_elems));
    cudaEventRecord(e0, c->stream);
    const int used = ws_predict_into(c, tmp + kLeadPad);
    cudaEventRecord(e1, c->stream);
    c->ws = saved;
    WS_CK(cudaStreamSynchronize(c->stream));
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    if (ms) *ms = t;
    int rc = TEA_OK;
    if (!used) {
        set_status(TEA_ERR_BAD_ARGUMENT, "tea_ws_predict_: chunk sides must be multiples of %d",
                   1 << (N->levels - 1));
        rc = TEA_ERR_BAD_ARGUMENT;
    } else if (du) {
        std::vector<double> u(c->field_elems), u0(c->field_elems);
        copy_on(c->stream, u.data(), tmp, sizeof(double) * c->field_elems, cudaMemcpyDeviceToHost);
        copy_on(c->stream, u0.data(), c->alloc[F_U0], sizeof(double) * c->field_elems, cudaMemcpyDeviceToHost);
        for (long i = 0; i < pix; ++i) {
            const long r = i / g.nx;
            const long f = kLeadPad + fidx(g, HALO_PAD + (int)(i % g.nx), HALO_PAD + (int)(r % g.ny),
                                           WS_3D ? HALO_PAD + (int)(r / g.ny) : 0);
            du[i] = u[f] - u0[f];
        }
    }
    cudaFree(tmp);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc == TEA_OK) rc = check_err(N, "predict");
    return rc;
}
