// Per-call device kernels behind the reference's ext_* entry points.  Each kernel states
// the functor(s) it replaces (crtrott/TeaLeaf-Kokkos tealeaf_2d|3d/ext_*.hpp); every
// expression keeps the reference's evaluation order so that, with -fmad=false, each
// stored value is bit-identical to the reference's.  Reductions are double-double
// (tea_common.cuh) and therefore match the oracle's compensated mode bit for bit.
//
// Unlike the reference (one thread per padded index, most masked off by a region test),
// each kernel walks only its region in 32 x 8 tiles with a grid-stride loop sized to the
// SM count; the halo is read from memory, as the reference reads it, so the per-call
// path also serves chunks whose halos hold a neighbour's data.
#pragma once

#include "tea_chunk.cuh"

namespace tea {

// SMVP(a), tealeaf_2d/ext_shared.hpp:37-41 / tealeaf_3d/ext_shared.hpp:39-45, with the
// reference's dims.x (row length) replaced by the row pitch and dims.x*dims.y by the page.
__device__ __forceinline__ double smvp(const double* __restrict__ a, const double* __restrict__ kx,
                                       const double* __restrict__ ky, const double* __restrict__ kz,
                                       long i, long pitch, long page)
{
#if TEA_DIM == 2
    (void)kz;
    (void)page;
    return (1.0 + (kx[i + 1] + kx[i]) + (ky[i + pitch] + ky[i])) * a[i]
        - (kx[i + 1] * a[i + 1] + kx[i] * a[i - 1])
        - (ky[i + pitch] * a[i + pitch] + ky[i] * a[i - pitch]);
#else
    return (1.0 + (kx[i + 1] + kx[i]) + (ky[i + pitch] + ky[i]) + (kz[i + page] + kz[i])) * a[i]
        - (kx[i + 1] * a[i + 1] + kx[i] * a[i - 1])
        - (ky[i + pitch] * a[i + pitch] + ky[i] * a[i - pitch])
        - (kz[i + page] * a[i + page] + kz[i] * a[i - page]);
#endif
}

// Diagonal of the operator (the preconditioner's 1/Mi), tealeaf_2d/ext_cg_kernel.hpp:119-121.
__device__ __forceinline__ double diag(const double* __restrict__ kx, const double* __restrict__ ky,
                                       const double* __restrict__ kz, long i, long pitch, long page)
{
#if TEA_DIM == 2
    (void)kz;
    (void)page;
    return (1.0 + (kx[i + 1] + kx[i]) + (ky[i + pitch] + ky[i]));
#else
    return (1.0 + (kx[i + 1] + kx[i]) + (ky[i + pitch] + ky[i]) + (kz[i + page] + kz[i]));
#endif
}

// Pointwise kernels walk the inner domain in row segments of 64 cells: a warp per segment,
// two adjacent cells per lane with one 16-byte access per array (the first inner cell of a
// row is 256-byte aligned, so column 2 + 2*lane is 16-byte aligned).  f(i, two) gets the
// lane's first cell and whether the second one is inner too.  Launched with 256-thread
// blocks (pair_blocks on the host).
template <class F>
__device__ __forceinline__ void walk_cell_pairs(const Geom& g, F&& f)
{
    const int per_row = (g.nx + 63) / 64;
    const long nseg = (long)per_row * g.ny * g.nz;
    const int lane = threadIdx.x & 31;
    const long warp0 = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long nwarps = ((long)gridDim.x * blockDim.x) >> 5;
    const int xlast = g.X - HALO_PAD - 1;
    for (long sgi = warp0; sgi < nseg; sgi += nwarps) {
        const long row = sgi / per_row;
        const int xs = (int)(sgi - row * per_row);
        const int jj = HALO_PAD + (int)(row % g.ny);
        const int ii = TEA_DIM == 3 ? HALO_PAD + (int)(row / g.ny) : 0;
        const int kk = HALO_PAD + xs * 64 + 2 * lane;
        if (kk <= xlast) f(fidx(g, kk, jj, ii), kk < xlast);
    }
}

__device__ __forceinline__ double2 ldp(const double* p) { return *reinterpret_cast<const double2*>(p); }
__device__ __forceinline__ void stp(double* p, double a, double b) { *reinterpret_cast<double2*>(p) = make_double2(a, b); }

// The operator at a lane's pair of cells (walk_cell_pairs): the operand at the cells and
// their neighbours, read from memory (halos included), and the face coefficients, with the
// pair's rows loaded as 16-byte vectors.  smvp_at(q) evaluates smvp() of cell i + q with the
// same operations in the same order.
struct Stencil2 {
    double c[2], xm[2], xp[2], ym[2], yp[2], zm[2], zp[2];
    double kx0[2], kx1[2], ky0[2], ky1[2], kz0[2], kz1[2];
    __device__ __forceinline__ void load(const Geom& g, const double* __restrict__ a, const double* __restrict__ kx,
                                         const double* __restrict__ ky, const double* __restrict__ kz, long i, bool two)
    {
        const long P = g.pitch;
        if (two) {
            const double2 cc = ldp(a + i), m = ldp(a + i - P), pp = ldp(a + i + P);
            const double l = a[i - 1], r = a[i + 2];
            c[0] = cc.x; c[1] = cc.y;
            xm[0] = l; xm[1] = cc.x;
            xp[0] = cc.y; xp[1] = r;
            ym[0] = m.x; ym[1] = m.y;
            yp[0] = pp.x; yp[1] = pp.y;
            const double2 k = ldp(kx + i);
            kx0[0] = k.x; kx0[1] = k.y;
            kx1[0] = k.y; kx1[1] = kx[i + 2];
            const double2 k0 = ldp(ky + i), k1 = ldp(ky + i + P);
            ky0[0] = k0.x; ky0[1] = k0.y;
            ky1[0] = k1.x; ky1[1] = k1.y;
#if TEA_DIM == 3
            const long Q = g.page;
            const double2 zm2 = ldp(a + i - Q), zp2 = ldp(a + i + Q), z0 = ldp(kz + i), z1 = ldp(kz + i + Q);
            zm[0] = zm2.x; zm[1] = zm2.y;
            zp[0] = zp2.x; zp[1] = zp2.y;
            kz0[0] = z0.x; kz0[1] = z0.y;
            kz1[0] = z1.x; kz1[1] = z1.y;
#endif
        } else {
            c[0] = a[i];
            xm[0] = a[i - 1];
            xp[0] = a[i + 1];
            ym[0] = a[i - P];
            yp[0] = a[i + P];
            kx0[0] = kx[i];
            kx1[0] = kx[i + 1];
            ky0[0] = ky[i];
            ky1[0] = ky[i + P];
#if TEA_DIM == 3
            const long Q = g.page;
            zm[0] = a[i - Q];
            zp[0] = a[i + Q];
            kz0[0] = kz[i];
            kz1[0] = kz[i + Q];
#endif
        }
    }
    __device__ __forceinline__ double smvp_at(int q) const
    {
#if TEA_DIM == 2
        return (1.0 + (kx1[q] + kx0[q]) + (ky1[q] + ky0[q])) * c[q] - (kx1[q] * xp[q] + kx0[q] * xm[q])
            - (ky1[q] * yp[q] + ky0[q] * ym[q]);
#else
        return (1.0 + (kx1[q] + kx0[q]) + (ky1[q] + ky0[q]) + (kz1[q] + kz0[q])) * c[q]
            - (kx1[q] * xp[q] + kx0[q] * xm[q]) - (ky1[q] * yp[q] + ky0[q] * ym[q])
            - (kz1[q] * zp[q] + kz0[q] * zm[q]);
#endif
    }
};

// ---------------------------------------------------------------- set-up

// InitialiseChunkAreas, tealeaf_2d/ext_initialise_chunk.hpp:63-90 (3D :66-99): volume only
// (the face areas are never read by any kernel).
__global__ void __launch_bounds__(BLOCK) k_init_volume(Geom g, Box full, double* volume, double v)
{
    walk(full, [&](int kk, int jj, int ii) { volume[fidx(g, kk, jj, ii)] = v; });
}

struct StateTable {
    int n, rect, circ, point;
    const double *density, *energy, *xmin, *xmax, *ymin, *ymax, *zmin, *zmax, *radius;
    const int* geometry;
};

// GenerateChunk, tealeaf_2d/ext_generate_chunk.hpp:13-101 (3D :13-109).
__global__ void __launch_bounds__(BLOCK) k_generate(Geom g, Box full, Fields f, StateTable s,
                                                    const double* __restrict__ vx,
                                                    const double* __restrict__ vy,
                                                    const double* __restrict__ vz,
                                                    const double* __restrict__ cx,
                                                    const double* __restrict__ cy,
                                                    const double* __restrict__ cz)
{
    walk(full, [&](int kk, int jj, int ii) {
        const long i = fidx(g, kk, jj, ii);
        double e0 = s.energy[0], den = s.density[0];
        for (int ss = 1; ss < s.n; ++ss) {
            bool apply = false;
            const int geo = s.geometry[ss];
            if (geo == s.rect) {
                apply = vx[kk + 1] >= s.xmin[ss] && vx[kk] < s.xmax[ss] && vy[jj + 1] >= s.ymin[ss]
                    && vy[jj] < s.ymax[ss];
#if TEA_DIM == 3
                apply = apply && vz[ii + 1] >= s.zmin[ss] && vz[ii] < s.zmax[ss];
#endif
            } else if (geo == s.circ) {
#if TEA_DIM == 2
                const double radius = sqrt((cx[kk] - s.xmin[ss]) * (cx[kk] - s.xmin[ss])
                                           + (cy[jj] - s.ymin[ss]) * (cy[jj] - s.ymin[ss]));
#else
                const double radius = sqrt((cx[kk] - s.xmin[ss]) * (cx[kk] - s.xmin[ss])
                                           + (cy[jj] - s.ymin[ss]) * (cy[jj] - s.ymin[ss])
                                           + (cz[ii] - s.zmin[ss]) * (cz[ii] - s.zmin[ss]));
#endif
                apply = radius <= s.radius[ss];
            } else if (geo == s.point) {
                apply = vx[kk] == s.xmin[ss] && vy[jj] == s.ymin[ss];
#if TEA_DIM == 3
                apply = apply && vz[ii] == s.zmin[ss];
#endif
            }
            if (apply) {
                e0 = s.energy[ss];
                den = s.density[ss];
            }
        }
        f.energy0[i] = e0;
        f.density[i] = den;
        bool one = kk > 0 && kk < g.X - 1 && jj > 0 && jj < g.Y - 1;
#if TEA_DIM == 3
        one = one && ii > 0 && ii < g.Z - 1;
#endif
        if (one) f.u[i] = e0 * den;
    });
    (void)vz;
    (void)cz;
}

// FieldSummary, tealeaf_2d/ext_field_summary.hpp:13-67.
__global__ void __launch_bounds__(BLOCK) k_field_summary(Geom g, Box inner, Fields f, RedScratch rs,
                                                         double* out)
{
    DDVec<4> acc;
    acc.zero();
    walk(inner, [&](int kk, int jj, int ii) {
        const long i = fidx(g, kk, jj, ii);
        const double cellVol = f.volume[i];
        const double cellMass = cellVol * f.density[i];
        dd_add(acc.v[0], cellVol);
        dd_add(acc.v[1], cellMass);
        dd_add(acc.v[2], cellMass * f.energy0[i]);
        dd_add(acc.v[3], cellMass * f.u[i]);
    });
    grid_reduce<4>(acc, rs, out);
}

// ---------------------------------------------------------------- halo and packing

// One reflective face update: halo[HALO_PAD-1-f] = interior[HALO_PAD+f].
struct HaloSeg {
    double* field;
    int face;   // 1 left, 2 right, 3 bottom, 4 top, 5 back, 6 front
    long count;
};

struct HaloJob {
    HaloSeg seg[36];
    int nseg;
    int depth;
};

// UpdateHalo, tealeaf_2d/ext_update_halo.hpp:12-76 (3D :12-136).  2D faces span the whole
// padded row/column; 3D faces only their inner part.  Within a face no element is both
// read and written, so the result does not depend on the thread mapping.
__global__ void k_update_halo(Geom g, HaloJob job)
{
    const HaloSeg sg = job.seg[blockIdx.y];
    const int depth = job.depth;
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < sg.count;
         idx += (long)gridDim.x * blockDim.x) {
        long to, from;
#if TEA_DIM == 2
        if (sg.face == 1 || sg.face == 2) {
            const int jj = (int)(idx / depth), fl = (int)(idx % depth);
            const int kt = sg.face == 1 ? HALO_PAD - 1 - fl : g.X - HALO_PAD + fl;
            const int kf = sg.face == 1 ? HALO_PAD + fl : g.X - HALO_PAD - 1 - fl;
            to = fidx(g, kt, jj, 0);
            from = fidx(g, kf, jj, 0);
        } else {
            const int kk = (int)(idx % g.X), fl = (int)(idx / g.X);
            const int jt = sg.face == 3 ? HALO_PAD - 1 - fl : g.Y - HALO_PAD + fl;
            const int jf = sg.face == 3 ? HALO_PAD + fl : g.Y - HALO_PAD - 1 - fl;
            to = fidx(g, kk, jt, 0);
            from = fidx(g, kk, jf, 0);
        }
#else
        if (sg.face == 1 || sg.face == 2) {
            const int fl = (int)(idx % depth);
            const long line = idx / depth;
            const int jj = HALO_PAD + (int)(line % g.ny), ii = HALO_PAD + (int)(line / g.ny);
            const int kt = sg.face == 1 ? HALO_PAD - 1 - fl : g.X - HALO_PAD + fl;
            const int kf = sg.face == 1 ? HALO_PAD + fl : g.X - HALO_PAD - 1 - fl;
            to = fidx(g, kt, jj, ii);
            from = fidx(g, kf, jj, ii);
        } else if (sg.face == 3 || sg.face == 4) {
            const int kk = HALO_PAD + (int)(idx % g.nx);
            const long line = idx / g.nx;
            const int fl = (int)(line % depth), ii = HALO_PAD + (int)(line / depth);
            const int jt = sg.face == 3 ? HALO_PAD - 1 - fl : g.Y - HALO_PAD + fl;
            const int jf = sg.face == 3 ? HALO_PAD + fl : g.Y - HALO_PAD - 1 - fl;
            to = fidx(g, kk, jt, ii);
            from = fidx(g, kk, jf, ii);
        } else {
            const int kk = HALO_PAD + (int)(idx % g.nx);
            const long line = idx / g.nx;
            const int jj = HALO_PAD + (int)(line % g.ny), fl = (int)(line / g.ny);
            const int it = sg.face == 5 ? HALO_PAD - 1 - fl : g.Z - HALO_PAD + fl;
            const int iF = sg.face == 5 ? HALO_PAD + fl : g.Z - HALO_PAD - 1 - fl;
            to = fidx(g, kk, jj, it);
            from = fidx(g, kk, jj, iF);
        }
#endif
        sg.field[to] = sg.field[from];
    }
}

// Packers, tealeaf_2d/ext_pack_kernel.hpp:8-97 and tealeaf_3d/ext_pack_kernel.hpp: the
// padded flat index of buffer element `index`, restated from each packer's offset
// expression, then mapped to the pitched layout.
// exact: the 2D bottom/top faces cover the inner columns 2..nx+1 (the reference's packer
// starts at column 0, tealeaf_2d/ext_pack_kernel.hpp:17-44; every other face is the same).
__device__ __forceinline__ long pack_flat_index(const Geom& g, int face, int depth, bool pack, long index,
                                                bool exact = false)
{
    const long X = g.X, Y = g.Y;
#if TEA_DIM == 2
    if (face == 1 || face == 2) {
        const long lines = index / depth;
        long off;
        if (face == 1) off = pack ? HALO_PAD + lines * (X - depth) : HALO_PAD - depth + lines * (X - depth);
        else off = pack ? X - HALO_PAD - depth + lines * (X - depth) : X - HALO_PAD + lines * (X - depth);
        return off + index;
    }
    const long width = X - 2 * HALO_PAD;
    const long lines = index / width;
    long off;
    if (face == 4) off = pack ? X * (Y - HALO_PAD - depth) + lines * 2 * HALO_PAD : X * (Y - HALO_PAD) + lines * 2 * HALO_PAD;
    else off = pack ? X * HALO_PAD + lines * 2 * HALO_PAD : X * (HALO_PAD - depth) + lines * 2 * HALO_PAD;
    return off + index + (exact ? HALO_PAD : 0);
#else
    const long Z = g.Z, HP2 = 2 * HALO_PAD, page = X * Y;
    if (face == 1 || face == 2) {
        const long height = Y - HP2;
        const long lines = index / depth;
        const long base = page * HALO_PAD + X * HALO_PAD + lines * (X - depth) + (lines / height) * X * HP2;
        long xoff;
        if (face == 1) xoff = pack ? HALO_PAD : HALO_PAD - depth;
        else xoff = pack ? X - HALO_PAD - depth : X - HALO_PAD;
        return base + xoff + index;
    }
    if (face == 3 || face == 4) {
        const long width = X - HP2;
        const long lines = index / width;
        long yoff;
        if (face == 4) yoff = pack ? X * (Y - HALO_PAD - depth) : X * (Y - HALO_PAD);
        else yoff = pack ? X * HALO_PAD : X * (HALO_PAD - depth);
        return page * HALO_PAD + yoff + HALO_PAD + lines * HP2 + X * (Y - depth) * (lines / depth) + index;
    }
    const long height = Y - HP2;
    const long lines = index / (X - HP2);
    long zoff;
    if (face == 6) zoff = pack ? page * (Z - HALO_PAD - depth) : page * (Z - HALO_PAD);
    else zoff = pack ? page * HALO_PAD : page * (HALO_PAD - depth);
    return zoff + X * HALO_PAD + HALO_PAD + lines * HP2 + (lines / height) * X * HP2 + index;
#endif
}

__global__ void k_pack(Geom g, double* field, double* buf, long len, int face, int depth, int pack, int exact)
{
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < len; idx += (long)gridDim.x * blockDim.x) {
        const long flat = pack_flat_index(g, face, depth, pack != 0, idx, exact != 0);
        const long kk = flat % g.X;
        const long rest = flat / g.X;
        const long jj = rest % g.Y;
        const long ii = rest / g.Y;
        const long p = fidx(g, (int)kk, (int)jj, (int)ii);
        if (pack) buf[idx] = field[p];
        else field[p] = buf[idx];
    }
}

// ---------------------------------------------------------------- shared solver methods

// SetField, tealeaf_2d/ext_set_field.hpp:13-29.
__global__ void __launch_bounds__(BLOCK) k_set_field(Geom g, Box full, Fields f)
{
    walk(full, [&](int kk, int jj, int ii) {
        const long i = fidx(g, kk, jj, ii);
        f.energy[i] = f.energy0[i];
    });
}

// CopyU, tealeaf_2d/ext_solver_methods.hpp:12-35.
__global__ void __launch_bounds__(BLOCK) k_copy_u(Geom g, Fields f)
{
    walk_cell_pairs(g, [&](long i, bool two) {
        if (two) {
            const double2 u = ldp(f.u + i);
            stp(f.u0 + i, u.x, u.y);
        } else {
            f.u0[i] = f.u[i];
        }
    });
}

// CalculateResidual, tealeaf_2d/ext_solver_methods.hpp:38-66.
__global__ void __launch_bounds__(BLOCK) k_residual(Geom g, Fields f)
{
    walk_cell_pairs(g, [&](long i, bool two) {
        Stencil2 n;
        n.load(g, f.u, f.kx, f.ky, f.kz, i, two);
        if (two) {
            const double2 u0 = ldp(f.u0 + i);
            stp(f.r + i, u0.x - n.smvp_at(0), u0.y - n.smvp_at(1));
        } else {
            f.r[i] = f.u0[i] - n.smvp_at(0);
        }
    });
}

// Calculate2Norm, tealeaf_2d/ext_solver_methods.hpp:70-92.
__global__ void __launch_bounds__(BLOCK) k_2norm(Geom g, const double* __restrict__ b, RedScratch rs, double* out)
{
    DDVec<1> acc;
    acc.zero();
    walk_cell_pairs(g, [&](long i, bool two) {
        if (two) {
            const double2 v = ldp(b + i);
            dd_add(acc.v[0], v.x * v.x);
            dd_add(acc.v[0], v.y * v.y);
        } else {
            const double v = b[i];
            dd_add(acc.v[0], v * v);
        }
    });
    grid_reduce<1>(acc, rs, out);
}

// Finalise, tealeaf_2d/ext_solver_methods.hpp:96-121.
__global__ void __launch_bounds__(BLOCK) k_finalise(Geom g, Fields f)
{
    walk_cell_pairs(g, [&](long i, bool two) {
        if (two) {
            const double2 u = ldp(f.u + i), d = ldp(f.density + i);
            stp(f.energy + i, u.x / d.x, u.y / d.y);
        } else {
            f.energy[i] = f.u[i] / f.density[i];
        }
    });
}

// ---------------------------------------------------------------- Jacobi

// JacobiInit, tealeaf_2d/ext_jacobi_kernel.hpp:12-62 (3D :12-66).
__global__ void __launch_bounds__(BLOCK) k_jacobi_init(Geom g, Box full, Fields f, int cond, double rx,
                                                       double ry, double rz)
{
    walk(full, [&](int kk, int jj, int ii) {
        const long i = fidx(g, kk, jj, ii);
        bool one = jj > 0 && jj < g.Y - 1 && kk > 0 && kk < g.X - 1;
        bool skew = jj >= HALO_PAD && jj < g.Y - 1 && kk >= HALO_PAD && kk < g.X - 1;
#if TEA_DIM == 3
        one = one && ii > 0 && ii < g.Z - 1;
        skew = skew && ii >= HALO_PAD && ii < g.Z - 1;
#endif
        if (one) {
            const double v = f.energy[i] * f.density[i];
            f.u0[i] = v;
            f.u[i] = v;
        }
        if (skew) {
            const double centre = cond ? f.density[i] : 1.0 / f.density[i];
            const double left = cond ? f.density[i - 1] : 1.0 / f.density[i - 1];
            const double down = cond ? f.density[i - g.pitch] : 1.0 / f.density[i - g.pitch];
            f.kx[i] = rx * (left + centre) / (2.0 * left * centre);
            f.ky[i] = ry * (down + centre) / (2.0 * down * centre);
#if TEA_DIM == 3
            const double back = cond ? f.density[i - g.page] : 1.0 / f.density[i - g.page];
            f.kz[i] = rz * (back + centre) / (2.0 * back * centre);
#endif
        }
    });
    (void)rz;
}

// JacobiCopyU, tealeaf_2d/ext_jacobi_kernel.hpp:66-82: r = u over the padded array.
__global__ void __launch_bounds__(BLOCK) k_jacobi_copy(Geom g, Fields f)
{
    // The whole padded array as one flat run of page * Z doubles (the pitch padding at the
    // end of each row is copied too; nothing reads it).  The array starts 16-byte aligned
    // and page is a multiple of 32, so every access is a 16-byte one.
    const long n2 = g.page * g.Z / 2;
    const double2* __restrict__ src = reinterpret_cast<const double2*>(f.u);
    double2* __restrict__ dst = reinterpret_cast<double2*>(f.r);
    for (long k = (long)blockIdx.x * blockDim.x + threadIdx.x; k < n2; k += (long)gridDim.x * blockDim.x)
        dst[k] = src[k];
}

// JacobiSolve, tealeaf_2d/ext_jacobi_kernel.hpp:86-117 (3D :90-126).
__global__ void __launch_bounds__(BLOCK) k_jacobi_solve(Geom g, Fields f, RedScratch rs, double* out)
{
    DDVec<1> acc;
    acc.zero();
    walk_cell_pairs(g, [&](long i, bool two) {
        Stencil2 n;
        n.load(g, f.r, f.kx, f.ky, f.kz, i, two);
        double u0[2], un[2];
        if (two) {
            const double2 v = ldp(f.u0 + i);
            u0[0] = v.x;
            u0[1] = v.y;
        } else {
            u0[0] = f.u0[i];
        }
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            if (q == 1 && !two) break;
#if TEA_DIM == 2
            un[q] = (u0[q] + (n.kx1[q] * n.xp[q] + n.kx0[q] * n.xm[q]) + (n.ky1[q] * n.yp[q] + n.ky0[q] * n.ym[q]))
                / (1.0 + (n.kx0[q] + n.kx1[q]) + (n.ky0[q] + n.ky1[q]));
#else
            un[q] = (u0[q] + (n.kx1[q] * n.xp[q] + n.kx0[q] * n.xm[q]) + (n.ky1[q] * n.yp[q] + n.ky0[q] * n.ym[q])
                     + (n.kz1[q] * n.zp[q] + n.kz0[q] * n.zm[q]))
                / (1.0 + (n.kx0[q] + n.kx1[q]) + (n.ky0[q] + n.ky1[q]) + (n.kz0[q] + n.kz1[q]));
#endif
            dd_add(acc.v[0], fabs(un[q] - n.c[q]));
        }
        if (two) stp(f.u + i, un[0], un[1]);
        else f.u[i] = un[0];
    });
    grid_reduce<1>(acc, rs, out);
}

// ---------------------------------------------------------------- CG

// CGInitU (tealeaf_2d/ext_cg_kernel.hpp:12-34) over the padded array, fused with CGInitW
// (:36-61) on the one-cell halo domain: both are pointwise.
__global__ void __launch_bounds__(BLOCK) k_cg_init_uw(Geom g, Box full, Fields f, int cond)
{
    walk(full, [&](int kk, int jj, int ii) {
        const long i = fidx(g, kk, jj, ii);
        f.p[i] = 0.0;
        f.r[i] = 0.0;
        f.u[i] = f.energy[i] * f.density[i];
        bool one = jj > 0 && jj < g.Y - 1 && kk > 0 && kk < g.X - 1;
#if TEA_DIM == 3
        one = one && ii > 0 && ii < g.Z - 1;
#endif
        if (one) f.w[i] = cond ? f.density[i] : 1.0 / f.density[i];
    });
}

// CGInitK, tealeaf_2d/ext_cg_kernel.hpp:63-91 (3D :59-91), on the skew domain.
__global__ void __launch_bounds__(BLOCK) k_cg_init_k(Geom g, Box skew, Fields f, double rx, double ry,
                                                     double rz)
{
    walk(skew, [&](int kk, int jj, int ii) {
        const long i = fidx(g, kk, jj, ii);
        const double* __restrict__ w = f.w;
        f.kx[i] = rx * (w[i - 1] + w[i]) / (2.0 * w[i - 1] * w[i]);
        f.ky[i] = ry * (w[i - g.pitch] + w[i]) / (2.0 * w[i - g.pitch] * w[i]);
#if TEA_DIM == 3
        f.kz[i] = rz * (w[i - g.page] + w[i]) / (2.0 * w[i - g.page] * w[i]);
#endif
    });
    (void)rz;
}

// CGCalcRRO, tealeaf_2d/ext_cg_kernel.hpp:93-145 (3D :93-149).
__global__ void __launch_bounds__(BLOCK) k_cg_calc_rro(Geom g, Box inner, Fields f, int precond,
                                                       RedScratch rs, double* out)
{
    DDVec<1> acc;
    acc.zero();
    walk(inner, [&](int kk, int jj, int ii) {
        const long i = fidx(g, kk, jj, ii);
        const double w = smvp(f.u, f.kx, f.ky, f.kz, i, g.pitch, g.page);
        f.w[i] = w;
        const double r = f.u[i] - w;
        f.r[i] = r;
        double p;
        if (precond) {
            const double mi = 1.0 / diag(f.kx, f.ky, f.kz, i, g.pitch, g.page);
            f.mi[i] = mi;
            const double z = mi * r;
            f.z[i] = z;
            p = z;
        } else {
            p = r;
        }
        f.p[i] = p;
        dd_add(acc.v[0], r * p);
    });
    grid_reduce<1>(acc, rs, out);
}

// CGCalcW, tealeaf_2d/ext_cg_kernel.hpp:148-197 (non-team operator, :177-189).
__global__ void __launch_bounds__(BLOCK) k_cg_calc_w(Geom g, Fields f, RedScratch rs, double* out)
{
    DDVec<1> acc;
    acc.zero();
    walk_cell_pairs(g, [&](long i, bool two) {
        Stencil2 n;
        n.load(g, f.p, f.kx, f.ky, f.kz, i, two);
        const double w0 = n.smvp_at(0);
        dd_add(acc.v[0], w0 * n.c[0]);
        if (two) {
            const double w1 = n.smvp_at(1);
            stp(f.w + i, w0, w1);
            dd_add(acc.v[0], w1 * n.c[1]);
        } else {
            f.w[i] = w0;
        }
    });
    grid_reduce<1>(acc, rs, out);
}

// CGCalcUr, tealeaf_2d/ext_cg_kernel.hpp:200-275 (non-team operator, :244-264).
__global__ void __launch_bounds__(BLOCK) k_cg_calc_ur(Geom g, Fields f, double alpha, int precond, RedScratch rs,
                                                      double* out)
{
    DDVec<1> acc;
    acc.zero();
    walk_cell_pairs(g, [&](long i, bool two) {
        if (two) {
            const double2 u = ldp(f.u + i), p = ldp(f.p + i), r = ldp(f.r + i), w = ldp(f.w + i);
            stp(f.u + i, u.x + alpha * p.x, u.y + alpha * p.y);
            const double r0 = r.x - alpha * w.x, r1 = r.y - alpha * w.y;
            stp(f.r + i, r0, r1);
            if (precond) {
                const double2 m = ldp(f.mi + i);
                const double z0 = m.x * r0, z1 = m.y * r1;
                stp(f.z + i, z0, z1);
                dd_add(acc.v[0], r0 * z0);
                dd_add(acc.v[0], r1 * z1);
            } else {
                dd_add(acc.v[0], r0 * r0);
                dd_add(acc.v[0], r1 * r1);
            }
        } else {
            f.u[i] = f.u[i] + alpha * f.p[i];
            const double r = f.r[i] - alpha * f.w[i];
            f.r[i] = r;
            if (precond) {
                const double z = f.mi[i] * r;
                f.z[i] = z;
                dd_add(acc.v[0], r * z);
            } else {
                dd_add(acc.v[0], r * r);
            }
        }
    });
    grid_reduce<1>(acc, rs, out);
}

// CGCalcP, tealeaf_2d/ext_cg_kernel.hpp:278-319 (non-team operator, :301-310).
__global__ void __launch_bounds__(BLOCK) k_cg_calc_p(Geom g, Fields f, double beta, int precond)
{
    const double* __restrict__ q = precond ? f.z : f.r;
    walk_cell_pairs(g, [&](long i, bool two) {
        if (two) {
            const double2 p = ldp(f.p + i), v = ldp(q + i);
            stp(f.p + i, beta * p.x + v.x, beta * p.y + v.y);
        } else {
            f.p[i] = beta * f.p[i] + q[i];
        }
    });
}

// ---------------------------------------------------------------- Chebyshev

// ChebyInit, tealeaf_2d/ext_cheby_kernel.hpp:11-47.
__global__ void __launch_bounds__(BLOCK) k_cheby_init(Geom g, Box inner, Fields f, double theta, int precond)
{
    walk(inner, [&](int kk, int jj, int ii) {
        const long i = fidx(g, kk, jj, ii);
        const double w = smvp(f.u, f.kx, f.ky, f.kz, i, g.pitch, g.page);
        f.w[i] = w;
        const double r = f.u0[i] - w;
        f.r[i] = r;
        f.p[i] = (precond ? f.mi[i] * r : r) / theta;
    });
}

// ChebyCalcU, tealeaf_2d/ext_cheby_kernel.hpp:50-72.
__global__ void __launch_bounds__(BLOCK) k_cheby_calc_u(Geom g, Fields f)
{
    walk_cell_pairs(g, [&](long i, bool two) {
        if (two) {
            const double2 u = ldp(f.u + i), p = ldp(f.p + i);
            stp(f.u + i, u.x + p.x, u.y + p.y);
        } else {
            f.u[i] = f.u[i] + f.p[i];
        }
    });
}

// ChebyIterate, tealeaf_2d/ext_cheby_kernel.hpp:75-115.
__global__ void __launch_bounds__(BLOCK) k_cheby_iterate(Geom g, Fields f, double alpha, double beta, int precond)
{
    walk_cell_pairs(g, [&](long i, bool two) {
        Stencil2 n;
        n.load(g, f.u, f.kx, f.ky, f.kz, i, two);
        if (two) {
            const double2 u0 = ldp(f.u0 + i), p = ldp(f.p + i);
            double2 m = make_double2(0.0, 0.0);
            if (precond) m = ldp(f.mi + i);
            const double w0 = n.smvp_at(0), w1 = n.smvp_at(1);
            stp(f.w + i, w0, w1);
            const double r0 = u0.x - w0, r1 = u0.y - w1;
            stp(f.r + i, r0, r1);
            stp(f.p + i, alpha * p.x + beta * (precond ? m.x * r0 : r0), alpha * p.y + beta * (precond ? m.y * r1 : r1));
        } else {
            const double w = n.smvp_at(0);
            f.w[i] = w;
            const double r = f.u0[i] - w;
            f.r[i] = r;
            f.p[i] = alpha * f.p[i] + beta * (precond ? f.mi[i] * r : r);
        }
    });
}

// ---------------------------------------------------------------- PPCG

// PPCGInitSd, tealeaf_2d/ext_ppcg_kernel.hpp:8-34.
__global__ void __launch_bounds__(BLOCK) k_ppcg_init_sd(Geom g, Fields f, double theta, int precond)
{
    walk_cell_pairs(g, [&](long i, bool two) {
        if (two) {
            const double2 r = ldp(f.r + i);
            double2 m = make_double2(0.0, 0.0);
            if (precond) m = ldp(f.mi + i);
            stp(f.sd + i, (precond ? m.x * r.x : r.x) / theta, (precond ? m.y * r.y : r.y) / theta);
        } else {
            f.sd[i] = (precond ? f.mi[i] * f.r[i] : f.r[i]) / theta;
        }
    });
}

// PPCGCalcU, tealeaf_2d/ext_ppcg_kernel.hpp:37-65.
__global__ void __launch_bounds__(BLOCK) k_ppcg_calc_u(Geom g, Fields f)
{
    walk_cell_pairs(g, [&](long i, bool two) {
        Stencil2 n;
        n.load(g, f.sd, f.kx, f.ky, f.kz, i, two);
        if (two) {
            const double2 r = ldp(f.r + i), u = ldp(f.u + i);
            stp(f.r + i, r.x - n.smvp_at(0), r.y - n.smvp_at(1));
            stp(f.u + i, u.x + n.c[0], u.y + n.c[1]);
        } else {
            f.r[i] = f.r[i] - n.smvp_at(0);
            f.u[i] = f.u[i] + n.c[0];
        }
    });
}

// PPCGCalcSd, tealeaf_2d/ext_ppcg_kernel.hpp:68-100.
__global__ void __launch_bounds__(BLOCK) k_ppcg_calc_sd(Geom g, Fields f, double alpha, double beta, int precond)
{
    walk_cell_pairs(g, [&](long i, bool two) {
        if (two) {
            const double2 sd = ldp(f.sd + i), r = ldp(f.r + i);
            double2 m = make_double2(0.0, 0.0);
            if (precond) m = ldp(f.mi + i);
            stp(f.sd + i, alpha * sd.x + beta * (precond ? m.x * r.x : r.x),
                alpha * sd.y + beta * (precond ? m.y * r.y : r.y));
        } else {
            f.sd[i] = alpha * f.sd[i] + beta * (precond ? f.mi[i] * f.r[i] : f.r[i]);
        }
    });
}

}  // namespace tea
