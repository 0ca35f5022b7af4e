// Element-wise, pooling, reduction and optimiser kernels of the learned warm-start network
// (no counterpart in the reference).  Shapes and conventions as in tea_ws_conv.cuh.
#pragma once

#include "tea_ws_conv.cuh"

namespace tea {
namespace ws {

struct View {  // a channel slice of a channels-last buffer
    bf16* p;
    int cs, co, c;  // channel stride, first channel, channels
};

// ----------------------------------------------------------------------------- weight gradient

// gW[co][t][ci] += sum_p gy[p][co] x[p + tap t][ci] and gb[co] += sum_p gy[p][co], float32
// accumulation on CUDA cores.  Block: one tap, a 32 x 32 (co, ci) tile and a slice of the
// pixels (blockIdx.y); 256 threads, each four (co, ci) products.
constexpr int WG_PIX = 64;

__global__ void __launch_bounds__(256) k_wgrad(const bf16* x, int xcs, int xco, const bf16* gy, int gcs, int gco,
                                                int n, int D, int H, int W, int cin, int cout, float* gw, float* gb)
{
    __shared__ float s_g[WG_PIX][33];
    __shared__ float s_x[WG_PIX][33];
    const int ci_tiles = (cin + 31) / 32, co_tiles = (cout + 31) / 32;
    int b = blockIdx.x;
    const int t = b % TAPS;
    b /= TAPS;
    const int cit = b % ci_tiles;
    const int cot = b / ci_tiles;
    if (cot >= co_tiles) return;
    const long npix = (long)n * D * H * W;
    const long per = (npix + gridDim.y - 1) / gridDim.y;
    const long pbeg = blockIdx.y * per, pend = min(npix, pbeg + per);
    const int tid = threadIdx.x;
    const int tco = tid >> 3;        // 0..31
    const int tci = (tid & 7) * 4;   // 0..28
    float acc[4] = {0.f, 0.f, 0.f, 0.f}, accb = 0.f;
    for (long p0 = pbeg; p0 < pend; p0 += WG_PIX) {
        for (int idx = tid; idx < WG_PIX * 32; idx += 256) {
            const int pp = idx / 32, c = idx % 32;
            const long p = p0 + pp;
            float gv = 0.f, xv = 0.f;
            if (p < pend) {
                const int co = cot * 32 + c;
                if (co < cout) gv = __bfloat162float(gy[p * gcs + gco + co]);
                const int ci = cit * 32 + c;
                if (ci < cin) {
                    const long sp = tap_src(pix_of(p, D, H, W), t, D, H, W);
                    if (sp >= 0) xv = __bfloat162float(x[sp * xcs + xco + ci]);
                }
            }
            s_g[pp][c] = gv;
            s_x[pp][c] = xv;
        }
        __syncthreads();
#pragma unroll 8
        for (int pp = 0; pp < WG_PIX; ++pp) {
            const float g = s_g[pp][tco];
            acc[0] += g * s_x[pp][tci];
            acc[1] += g * s_x[pp][tci + 1];
            acc[2] += g * s_x[pp][tci + 2];
            acc[3] += g * s_x[pp][tci + 3];
            accb += g;
        }
        __syncthreads();
    }
    const int co = cot * 32 + tco;
    if (co < cout) {
        for (int k = 0; k < 4; ++k) {
            const int ci = cit * 32 + tci + k;
            if (ci < cin) atomicAdd(&gw[((long)co * TAPS + t) * cin + ci], acc[k]);
        }
        if (gb && t == 0 && cit == 0 && tci == 0) atomicAdd(&gb[co], accb);
    }
}

// ----------------------------------------------------------------------------- pooling

// Each coarse pixel averages its 2^dim children (2x2 in 2D, 2x2x2 in 3D); upsampling copies
// it back to them.  D, H, W are the fine sizes (D = 1 in 2D).
constexpr int POOL = WS_3D ? 8 : 4;

__host__ __device__ __forceinline__ int coarse_d(int D) { return WS_3D ? D / 2 : 1; }

// Fine pixel of child c (bit 0: x, bit 1: y, bit 2: z) of coarse pixel q.
__device__ __forceinline__ long child_of(const Pix& q, int c, int D, int H, int W)
{
    const int fx = 2 * q.x + (c & 1), fy = 2 * q.y + ((c >> 1) & 1), fz = WS_3D ? 2 * q.z + ((c >> 2) & 1) : 0;
    return ((q.img * D + fz) * (long)H + fy) * W + fx;
}

// Coarse pixel of fine pixel p.
__device__ __forceinline__ long parent_of(long p, int D, int H, int W)
{
    const Pix f = pix_of(p, D, H, W);
    const int d2 = coarse_d(D);
    return ((f.img * d2 + (WS_3D ? f.z / 2 : 0)) * (long)(H / 2) + f.y / 2) * (W / 2) + f.x / 2;
}

// The pooling kernels take one pixel per thread and its channels 8 at a time (16-byte
// loads and stores: channel counts, strides and offsets are multiples of 8), so that a
// pixel's position is decoded once.
struct Vec8 {
    float v[8];
};

__device__ __forceinline__ Vec8 ld8(const bf16* p)
{
    Vec8 r;
    const uint4 u = *reinterpret_cast<const uint4*>(p);
    const bf16* b = reinterpret_cast<const bf16*>(&u);
#pragma unroll
    for (int k = 0; k < 8; ++k) r.v[k] = __bfloat162float(b[k]);
    return r;
}

__device__ __forceinline__ void st8(bf16* p, const Vec8& r)
{
    __align__(16) bf16 b[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) b[k] = __float2bfloat16(r.v[k]);
    *reinterpret_cast<uint4*>(p) = *reinterpret_cast<const uint4*>(b);
}

__global__ void k_avgpool(View x, bf16* y, int n, int D, int H, int W)
{
    const int d2 = coarse_d(D), h2 = H / 2, w2 = W / 2;
    const long total = (long)n * d2 * h2 * w2;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < total; q += (long)gridDim.x * blockDim.x) {
        const Pix qc = pix_of(q, d2, h2, w2);
        long ch[POOL];
#pragma unroll
        for (int d = 0; d < POOL; ++d) ch[d] = child_of(qc, d, D, H, W) * x.cs + x.co;
        for (int c = 0; c < x.c; c += 8) {
            Vec8 s;
#pragma unroll
            for (int k = 0; k < 8; ++k) s.v[k] = 0.f;
#pragma unroll
            for (int d = 0; d < POOL; ++d) {
                const Vec8 v = ld8(x.p + ch[d] + c);
#pragma unroll
                for (int k = 0; k < 8; ++k) s.v[k] += v.v[k];
            }
#pragma unroll
            for (int k = 0; k < 8; ++k) s.v[k] = s.v[k] * (1.0f / POOL);
            st8(y + q * x.c + c, s);
        }
    }
}

// g_fine = (g_coarse / 2^dim) * (act > 0) + g_skip, the gradient with respect to the
// pre-activation of an encoder level's last convolution.
__global__ void k_avgpool_bw(const bf16* gc, View act, View gskip, bf16* gf, int n, int D, int H, int W)
{
    const int C = act.c;
    const long total = (long)n * D * H * W;
    for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < total; p += (long)gridDim.x * blockDim.x) {
        const long q = parent_of(p, D, H, W);
        for (int c = 0; c < C; c += 8) {
            const Vec8 g = ld8(gc + q * C + c);
            const Vec8 a = ld8(act.p + p * act.cs + act.co + c);
            const Vec8 k = ld8(gskip.p + p * gskip.cs + gskip.co + c);
            Vec8 o;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                float v = (1.0f / POOL) * g.v[j];
                if (!(a.v[j] > 0.f)) v = 0.f;
                o.v[j] = v + k.v[j];
            }
            st8(gf + p * C + c, o);
        }
    }
}

__global__ void k_upsample(View h, View cat, int n, int D, int H, int W)  // D, H, W: fine size
{
    const int C = h.c;
    const long total = (long)n * D * H * W;
    for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < total; p += (long)gridDim.x * blockDim.x) {
        const long q = parent_of(p, D, H, W);
        for (int c = 0; c < C; c += 8)
            *reinterpret_cast<uint4*>(cat.p + p * cat.cs + cat.co + c) =
                *reinterpret_cast<const uint4*>(h.p + q * h.cs + h.co + c);
    }
}

__global__ void k_upsample_bw(View gcat, bf16* gh, int n, int D, int H, int W)  // D, H, W: fine size
{
    const int C = gcat.c, d2 = coarse_d(D), h2 = H / 2, w2 = W / 2;
    const long total = (long)n * d2 * h2 * w2;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < total; q += (long)gridDim.x * blockDim.x) {
        const Pix qc = pix_of(q, d2, h2, w2);
        long ch[POOL];
#pragma unroll
        for (int d = 0; d < POOL; ++d) ch[d] = child_of(qc, d, D, H, W) * gcat.cs + gcat.co;
        for (int c = 0; c < C; c += 8) {
            Vec8 s;
#pragma unroll
            for (int k = 0; k < 8; ++k) s.v[k] = 0.f;
#pragma unroll
            for (int d = 0; d < POOL; ++d) {
                const Vec8 v = ld8(gcat.p + ch[d] + c);
#pragma unroll
                for (int k = 0; k < 8; ++k) s.v[k] += v.v[k];
            }
            st8(gh + q * C + c, s);
        }
    }
}

// ----------------------------------------------------------------------------- head and loss

// y = h . w + b per pixel (float32 out).  With a target: sums[0] += (y - t)^2 and the
// backward pass: gy = 2 (y - t) / N, gh = gy w (h > 0), gw += gy h, gb += gy.
template <int C>
__global__ void __launch_bounds__(256) k_head(const bf16* h, const float* w, const float* b, float* y, long npix,
                                               const float* target, float* sums, bf16* gh, float* gw, float* gb)
{
    __shared__ float s_w[C];
    __shared__ float s_red[C + 2];
    for (int c = threadIdx.x; c < C; c += blockDim.x) s_w[c] = w[c];
    for (int c = threadIdx.x; c < C + 2; c += blockDim.x) s_red[c] = 0.f;
    __syncthreads();
    float gwl[C];
#pragma unroll
    for (int c = 0; c < C; ++c) gwl[c] = 0.f;
    float lossl = 0.f, gbl = 0.f;
    const float inv = 2.0f / (float)npix;
    for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < npix; p += (long)gridDim.x * blockDim.x) {
        float hv[C];
        float acc = b[0];
#pragma unroll
        for (int c = 0; c < C; ++c) {
            hv[c] = __bfloat162float(h[p * C + c]);
            acc += hv[c] * s_w[c];
        }
        y[p] = acc;
        if (target) {
            const float d = acc - target[p];
            lossl += d * d;
            const float g = inv * d;
            gbl += g;
#pragma unroll
            for (int c = 0; c < C; ++c) {
                gwl[c] += g * hv[c];
                gh[p * C + c] = __float2bfloat16(hv[c] > 0.f ? g * s_w[c] : 0.f);
            }
        }
    }
    if (!target) return;
#pragma unroll
    for (int c = 0; c < C; ++c) atomicAdd(&s_red[c], gwl[c]);
    atomicAdd(&s_red[C], gbl);
    atomicAdd(&s_red[C + 1], lossl);
    __syncthreads();
    for (int c = threadIdx.x; c < C; c += blockDim.x) atomicAdd(&gw[c], s_red[c]);
    if (threadIdx.x == 0) {
        atomicAdd(gb, s_red[C]);
        atomicAdd(&sums[0], s_red[C + 1]);
    }
}

// ----------------------------------------------------------------------------- residual loss

// The solver's operator on an n x [D x] H x W crop stack, A v = (1 + sum of the cell's
// face coefficients) v - sum K_face v_neighbour, with kk[NK p ..] = (Kx, Ky[, Kz]) of pixel
// p (the faces to its left, below [and behind]) and the crop's outer faces taken as zero
// (no flux), which keeps A symmetric.
constexpr int NK = WS_3D ? 3 : 2;

// The six (four) face coefficients of pixel q = p.
struct Faces {
    float xl, xr, yd, yu, zb, zf;
};

__device__ __forceinline__ Faces faces_of(const float* kk, long p, const Pix& q, int D, int H, int W)
{
    Faces f;
    const long page = (long)H * W;
    f.xl = q.x > 0 ? kk[NK * p] : 0.f;
    f.xr = q.x + 1 < W ? kk[NK * (p + 1)] : 0.f;
    f.yd = q.y > 0 ? kk[NK * p + 1] : 0.f;
    f.yu = q.y + 1 < H ? kk[NK * (p + W) + 1] : 0.f;
    f.zb = WS_3D && q.z > 0 ? kk[NK * p + 2] : 0.f;
    f.zf = WS_3D && q.z + 1 < D ? kk[NK * (p + page) + 2] : 0.f;
    return f;
}

__device__ __forceinline__ float diag_of(const Faces& f)
{
    return WS_3D ? 1.f + f.xl + f.xr + f.yd + f.yu + f.zb + f.zf : 1.f + f.xl + f.xr + f.yd + f.yu;
}

__device__ __forceinline__ float apply_a(const float* v, const float* kk, long p, const Pix& q, int D, int H, int W)
{
    const Faces f = faces_of(kk, p, q, D, H, W);
    float a = diag_of(f) * v[p];
    if (q.x > 0) a -= f.xl * v[p - 1];
    if (q.x + 1 < W) a -= f.xr * v[p + 1];
    if (q.y > 0) a -= f.yd * v[p - W];
    if (q.y + 1 < H) a -= f.yu * v[p + W];
    if (WS_3D) {
        const long page = (long)H * W;
        if (q.z > 0) a -= f.zb * v[p - page];
        if (q.z + 1 < D) a -= f.zf * v[p + page];
    }
    return a;
}

// Pass 0: d = y - t.  Pass 1 (d now the smoothed error): e = A d; per image b (blockIdx.y),
// sums[2b] += d.(A d) and sums[2b + 1] += t.(A t): the energy norm of the guess's error and
// that of the plain start's (du = 0).
__global__ void k_res_loss(const float* y, const float* t, const float* kk, float* d, float* e, int D, int H,
                           int W, float* sums, int pass)
{
    const long per = (long)D * H * W;
    const long off = (long)blockIdx.y * per;
    float s0 = 0.f, s1 = 0.f;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < per; q += (long)gridDim.x * blockDim.x) {
        const long p = off + q;
        if (pass == 0) {
            d[p] = y[p] - t[p];
        } else {
            const Pix pq = pix_of(q, D, H, W);
            const float ev = apply_a(d, kk, p, pq, D, H, W);
            e[p] = ev;
            s0 += d[p] * ev;
            s1 += t[p] * apply_a(t, kk, p, pq, D, H, W);
        }
    }
    if (pass == 0) return;
    __shared__ float r0[256], r1[256];
    r0[threadIdx.x] = s0;
    r1[threadIdx.x] = s1;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            r0[threadIdx.x] += r0[threadIdx.x + o];
            r1[threadIdx.x] += r1[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        atomicAdd(&sums[2 * blockIdx.y], r0[0]);
        atomicAdd(&sums[2 * blockIdx.y + 1], r1[0]);
    }
}

// dL/d(smoothed error) of L = (1/n) sum_b d_b.(A d_b) / t_b.(A t_b): 2 A d_b / (n t_b.(A t_b)),
// with e = A d from pass 1.
__global__ void k_res_grad(const float* e, const float* kk, const float* sums, float* gy, int n, int D, int H,
                           int W)
{
    const long per = (long)D * H * W;
    const long off = (long)blockIdx.y * per;
    // Crops with almost no activity (t.A t tiny) would dominate: their denominator is floored
    // at 1e-3 of the batch's largest.
    float dmax = 0.f;
    for (int b = 0; b < n; ++b) dmax = fmaxf(dmax, sums[2 * b + 1]);
    const float sc = 2.f / ((float)n * fmaxf(fmaxf(sums[2 * blockIdx.y + 1], 1e-3f * dmax), 1e-30f));
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < per; q += (long)gridDim.x * blockDim.x) {
        const long p = off + q;
        gy[p] = sc * e[p];
    }
    (void)kk;
    (void)W;
}

// The warm start smooths the network's guess with damped Jacobi sweeps in FP64 before the
// solve; training sees the same linear smoothing on the error e = y - t:
//   e <- M e,  M = I - omega D^-1 A        (forward),
//   g <- M^T g = g - omega A (D^-1 g)      (backward; A symmetric, D its diagonal).
constexpr int WS_SMOOTH = 8;
constexpr float WS_OMEGA = 0.8f;

// out = in - omega D^-1 A in (transpose = 0), or out = in - omega A tmp with tmp = D^-1 in
// precomputed (transpose = 1); over n images of [D x] H x W.
__global__ void k_smooth_err(const float* in, const float* tmp, float* out, const float* kk, int n, int D, int H,
                             int W, int transpose)
{
    const long total = (long)n * D * H * W;
    for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < total; p += (long)gridDim.x * blockDim.x) {
        const Pix q = pix_of(p, D, H, W);
        if (!transpose)
            out[p] = in[p] - WS_OMEGA * apply_a(in, kk, p, q, D, H, W) / diag_of(faces_of(kk, p, q, D, H, W));
        else
            out[p] = in[p] - WS_OMEGA * apply_a(tmp, kk, p, q, D, H, W);
    }
}

__global__ void k_dinv(const float* in, float* out, const float* kk, int n, int D, int H, int W)
{
    const long total = (long)n * D * H * W;
    for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < total; p += (long)gridDim.x * blockDim.x) {
        const Pix q = pix_of(p, D, H, W);
        out[p] = in[p] / diag_of(faces_of(kk, p, q, D, H, W));
    }
}

// Head backward from a given dL/dy: gh = gy w (h > 0), gw += gy h, gb += gy.
template <int C>
__global__ void __launch_bounds__(256) k_head_bw(const bf16* h, const float* w, const float* gy, long npix, bf16* gh,
                                                  float* gw, float* gb)
{
    __shared__ float s_w[C];
    __shared__ float s_red[C + 1];
    for (int c = threadIdx.x; c < C; c += blockDim.x) s_w[c] = w[c];
    for (int c = threadIdx.x; c < C + 1; c += blockDim.x) s_red[c] = 0.f;
    __syncthreads();
    float gwl[C];
#pragma unroll
    for (int c = 0; c < C; ++c) gwl[c] = 0.f;
    float gbl = 0.f;
    for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < npix; p += (long)gridDim.x * blockDim.x) {
        const float g = gy[p];
        gbl += g;
#pragma unroll
        for (int c = 0; c < C; ++c) {
            const float hv = __bfloat162float(h[p * C + c]);
            gwl[c] += g * hv;
            gh[p * C + c] = __float2bfloat16(hv > 0.f ? g * s_w[c] : 0.f);
        }
    }
#pragma unroll
    for (int c = 0; c < C; ++c) atomicAdd(&s_red[c], gwl[c]);
    atomicAdd(&s_red[C], gbl);
    __syncthreads();
    for (int c = threadIdx.x; c < C; c += blockDim.x) atomicAdd(&gw[c], s_red[c]);
    if (threadIdx.x == 0) atomicAdd(gb, s_red[C]);
}

// ----------------------------------------------------------------------------- optimiser

// Adam on float32 master weights; clears the gradient.
__global__ void k_adam(float* w, float* g, float* m, float* v, long count, float lr, float b1, float b2, float eps,
                       float c1, float c2)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < count; i += (long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        g[i] = 0.f;
    }
}

// bfloat16 copies of a layer: w16[co][t][ci] and, for the input gradient, the transposed,
// tap-flipped wt16[ci][t][co] = w[co][TAPS - 1 - t][ci] (every offset of the tap negated).
__global__ void k_weights_bf16(const float* w, bf16* w16, bf16* wt16, int cout, int cin)
{
    const long total = (long)cout * TAPS * cin;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const int ci = (int)(i % cin);
        const int t = (int)((i / cin) % TAPS);
        const int co = (int)(i / ((long)TAPS * cin));
        const bf16 v = __float2bfloat16(w[i]);
        w16[i] = v;
        if (wt16) wt16[((long)ci * TAPS + (TAPS - 1 - t)) * cout + co] = v;
    }
}

}  // namespace ws
}  // namespace tea
