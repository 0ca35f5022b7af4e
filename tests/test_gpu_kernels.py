"""Kernel-level parity of the CUDA library (libtea{2,3}d_b200.so) with the oracle.

Every ext_* entry point is called through the C ABI on identical random inputs in the
CUDA library and in the oracle (compensated sums, the order-independent mode the CUDA
library uses), and every field array -- halos included -- and every returned scalar must
be bit-identical.  Grids are small and deliberately ragged (not multiples of the tiles).
"""
import ctypes

import numpy as np
import pytest

from conftest import PORT, SUM_COMPENSATED, port_lib, tea

pytestmark = pytest.mark.gpu

SIZES = {2: [(37, 29, 1), (64, 64, 1), (130, 67, 1)], 3: [(13, 11, 9), (33, 17, 20)]}
ALL_FIELDS = ["density", "energy0", "energy1", "u", "p", "sd", "u0", "r", "w", "z", "mi", "kx", "ky", "volume"]


def fields_for(dim):
    return ALL_FIELDS + (["kz"] if dim == 3 else [])


class Pair:
    """The same chunk in the CUDA library and in the oracle."""

    def __init__(self, dim, nx, ny, nz, seed):
        self.dim = dim
        self.gpu_lib = tea.cuda_library(dim)
        port_lib(dim, SUM_COMPENSATED)
        self.cpu_lib = tea.load_library(PORT[dim])
        self.gpu = tea.ExtChunk(self.gpu_lib, dim, nx, ny, nz)
        self.cpu = tea.ExtChunk(self.cpu_lib, dim, nx, ny, nz)
        rng = np.random.default_rng(seed)
        shape = (self.gpu.Z, self.gpu.Y, self.gpu.X)
        for f in fields_for(dim):
            if f == "density":
                a = 10.0 ** rng.uniform(-1, 2, shape)
            elif f in ("kx", "ky", "kz"):
                a = rng.uniform(0.0, 3.0, shape)
            elif f == "mi":
                a = rng.uniform(0.1, 1.0, shape)
            else:
                a = rng.uniform(-1.0, 25.0, shape)
            self.gpu.write(f, a)
            self.cpu.write(f, a)
        for c in (self.gpu, self.cpu):
            c.initialise(0.0, 0.0, 10.0 / nx, 10.0 / ny, 0.0, 10.0 / max(nz, 1))

    def both(self, fn):
        return fn(self.gpu), fn(self.cpu)

    def check(self, what):
        for f in fields_for(self.dim):
            g, c = self.gpu.read(f), self.cpu.read(f)
            if not np.array_equal(g, c):
                bad = np.argwhere(g != c)
                i = tuple(bad[0])
                raise AssertionError(f"{what}: field {f} differs at {len(bad)} points, first {i}: "
                                     f"gpu {g[i]!r} oracle {c[i]!r}")

    def close(self):
        self.gpu_lib.ext_finalise_()
        self.cpu_lib.ext_finalise_()


def I(v):
    return ctypes.byref(ctypes.c_int(v))


def D(v):
    return ctypes.byref(ctypes.c_double(v))


@pytest.fixture(params=[(d, s) for d in (2, 3) for s in SIZES[d]], ids=lambda p: f"{p[0]}d-{'x'.join(map(str, p[1]))}")
def pair(request):
    dim, (nx, ny, nz) = request.param
    p = Pair(dim, nx, ny, nz, seed=nx * 1000 + ny)
    p.check("after write")
    yield p
    p.close()


def test_set_up_kernels(pair):
    d = pair.dim
    n = 5
    den = np.array([100.0, 0.1, 5.0, 2.0, 0.7])
    en = np.array([1e-4, 25.0, 3.0, 1.5, 9.0])
    x0 = np.array([0.0, 0.5, 6.0, 2.0, 3.3333333333333335])
    x1 = np.array([0.0, 2.0, 0.0, 7.0, 0.0])
    y0 = np.array([0.0, 1.0, 5.0, 3.0, 6.6666666666666670])
    y1 = np.array([0.0, 4.0, 0.0, 8.0, 0.0])
    z0 = np.array([0.0, 2.0, 5.0, 1.0, 0.0])
    z1 = np.array([0.0, 9.0, 0.0, 4.0, 0.0])
    rad = np.array([0.0, 0.0, 1.7, 0.0, 0.0])
    geo = np.array([0, 1, 2, 1, 3], dtype=np.int32)
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)

    def gen(c):
        if d == 2:
            c.call("ext_generate_chunk_", I(n), P(den), P(en), P(x0), P(x1), P(y0), P(y1), P(rad), P(geo),
                   I(1), I(2), I(3))
        else:
            c.call("ext_generate_chunk_", I(n), P(den), P(en), P(x0), P(x1), P(y0), P(y1), P(z0), P(z1), P(rad),
                   P(geo), I(1), I(2), I(3))
    pair.both(gen)
    pair.check("ext_generate_chunk_")
    pair.both(lambda c: c.call("ext_set_field_kernel_"))
    pair.check("ext_set_field_kernel_")
    g, c = pair.both(lambda c: c.field_summary())
    assert g == c


@pytest.mark.parametrize("depth", [1, 2])
def test_update_halo(pair, depth):
    nb = [-1] * 6
    pair.both(lambda c: c.update_halo({1, 2, 3, 4, 5, 6}, depth, nb))
    pair.check(f"halo depth {depth}")
    nb2 = [-1, 7, -1, 3, -1, 2]  # some faces internal: left untouched
    pair.both(lambda c: c.update_halo({4, 6}, depth, nb2))
    pair.check(f"halo depth {depth} partial")


@pytest.mark.parametrize("coef,precond", [(1, 0), (2, 0), (1, 1), (2, 1)])
def test_cg_sequence(pair, coef, precond):
    g, c = pair.both(lambda ch: ch.reduce("ext_cg_solver_init_", I(coef), I(precond), D(0.004)))
    assert g == c, (g, c)
    pair.check("ext_cg_solver_init_")
    pair.both(lambda ch: ch.update_halo({4, 5}, 1))
    g, c = pair.both(lambda ch: ch.reduce("ext_cg_calc_w_"))
    assert g == c
    pair.check("ext_cg_calc_w_")
    alpha = g and (1.0 / 3.0)
    g, c = pair.both(lambda ch: ch.reduce("ext_cg_calc_ur_", D(0.37)))
    assert g == c
    pair.check("ext_cg_calc_ur_")
    pair.both(lambda ch: ch.call("ext_cg_calc_p_", D(0.61)))
    pair.check("ext_cg_calc_p_")
    del alpha


@pytest.mark.parametrize("precond", [0, 1])
def test_chebyshev_and_ppcg(pair, precond):
    pair.both(lambda ch: ch.reduce("ext_cg_solver_init_", I(2), I(precond), D(0.004)))
    n = 12
    al = np.linspace(0.3, 0.9, n)
    be = np.linspace(1.1, 0.2, n)
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    pair.both(lambda ch: ch.call("ext_cheby_solver_init_", P(al), P(be), D(0.75), I(precond), I(n)))
    pair.check("ext_cheby_solver_init_")
    for step in (n, 2, 3):
        pair.both(lambda ch: ch.update_halo({4}, 1))
        pair.both(lambda ch: ch.call("ext_cheby_solver_iterate_", I(step)))
        pair.check(f"ext_cheby_solver_iterate_ {step}")
    pair.both(lambda ch: ch.call("ext_ppcg_init_", P(al), P(be), D(1.25), I(n)))
    pair.both(lambda ch: ch.call("ext_calculate_residual_"))
    pair.check("ext_calculate_residual_")
    pair.both(lambda ch: ch.call("ext_ppcg_init_sd_"))
    pair.check("ext_ppcg_init_sd_")
    for k in range(1, 5):
        pair.both(lambda ch: ch.update_halo({6}, 1))
        pair.both(lambda ch: ch.call("ext_ppcg_inner_", I(k)))
        pair.check(f"ext_ppcg_inner_ {k}")
    for flag in (1, 0):
        g, c = pair.both(lambda ch: ch.norm2(flag))
        assert g == c


@pytest.mark.parametrize("coef", [1, 2])
def test_jacobi_and_methods(pair, coef):
    pair.both(lambda ch: ch.call("ext_jacobi_kernel_init_", I(coef), D(0.004)))
    pair.check("ext_jacobi_kernel_init_")
    for it in range(3):
        g, c = pair.both(lambda ch: ch.reduce("ext_jacobi_kernel_solve_"))
        assert g == c
        pair.check(f"ext_jacobi_kernel_solve_ {it}")
        pair.both(lambda ch: ch.update_halo({4}, 1))
    pair.both(lambda ch: ch.call("ext_solver_copy_u_"))
    pair.both(lambda ch: ch.call("ext_calculate_residual_"))
    pair.both(lambda ch: ch.call("ext_solver_finalise_"))
    pair.check("copy_u/residual/finalise")
    g, c = pair.both(lambda ch: ch.field_summary())
    assert g == c


@pytest.mark.parametrize("packer", ["ext_pack_message_", "tea_pack_face_"])
def test_pack_message(pair, packer):
    d = pair.dim
    faces = [1, 2, 3, 4] + ([5, 6] if d == 3 else [])
    nx, ny, nz = pair.gpu.X - 4, pair.gpu.Y - 4, max(pair.gpu.Z - 4, 1)
    field_type = [I(1)] if d == 3 and packer == "ext_pack_message_" else []
    for face in faces:
        for depth in (1, 2):
            if face <= 2:
                n = ny * (nz if d == 3 else 1) * depth
            elif face <= 4:
                n = nx * (nz if d == 3 else 1) * depth
            else:
                n = nx * ny * depth
            fields = (ctypes.c_int * 6)(1, 0, 1, 1, 0, 1)
            offsets = (ctypes.c_int * 6)(*[k * n for k in range(6)])
            bufs = {}
            for name, ch in (("gpu", pair.gpu), ("cpu", pair.cpu)):
                buf = np.zeros(6 * n)
                args = [fields, offsets, I(depth), I(face)] + field_type
                ch.call(packer, *args, buf.ctypes.data_as(ctypes.c_void_p), I(1))
                bufs[name] = buf
            assert np.array_equal(bufs["gpu"], bufs["cpu"]), (face, depth)
            src = np.arange(6 * n, dtype=np.float64) * 0.5
            for ch in (pair.gpu, pair.cpu):
                args = [fields, offsets, I(depth), I(face)] + field_type
                ch.call(packer, *args, src.ctypes.data_as(ctypes.c_void_p), I(0))
            pair.check(f"unpack face {face} depth {depth}")
