"""TeaLeaf implicit heat-conduction solve on one B200 -- host-side Python mirror.

The product is native: ``libtea2d_b200.so`` / ``libtea3d_b200.so`` export the reference's
``ext_*`` C ABI (include/tea_ext_2d.h, include/tea_ext_3d.h) backed by sm_100a CUDA,
and ``libtea_driver.so`` is the C++ restatement of the reference's Fortran driver that
runs a ``tea.in`` deck against that ABI.  This module only binds them with ctypes:

* :func:`run_deck` -- run a deck through the driver (the reference's ``tea_leaf``
  executable, ``tealeaf_2d/tea_leaf.f90``), returning the run summary and per-step
  records (iteration counts, errors, field summaries).
* :class:`ExtChunk` -- call individual ``ext_*`` entry points on one chunk and read or
  write its fields, for kernel-level checks.
* :func:`seeded_deck` -- the seeded synthetic state generator that writes standard
  ``tea.in`` decks.

There is no CPU fallback: loading a library that is missing raises, and on a machine
without a GPU the CUDA library reports ``TEA_ERR_NO_DEVICE`` at ``ext_init_``.
"""
from __future__ import annotations

import ctypes
import math
import os
import pathlib
from dataclasses import dataclass

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent

FIELD_IDS = {
    "density": 1, "energy0": 2, "energy1": 3, "u": 4, "p": 5, "sd": 6, "u0": 7, "r": 8,
    "w": 9, "z": 10, "mi": 11, "kx": 12, "ky": 13, "kz": 14, "volume": 15,
}
SOLVERS = {"jacobi": 1, "cg": 2, "chebyshev": 3, "ppcg": 4}
PRECISION_FP64, PRECISION_FP32_REFINED = 0, 1
SOLVER_KEYWORDS = {1: "tl_use_jacobi", 2: "tl_use_cg", 3: "tl_use_chebyshev", 4: "tl_use_ppcg"}


def lib_path(dim: int) -> pathlib.Path:
    """Path of the CUDA library for ``dim`` (2 or 3)."""
    return HERE / f"libtea{dim}d_b200.so"


def driver_path() -> pathlib.Path:
    return HERE / "libtea_driver.so"


def tea_leaf_exe() -> pathlib.Path:
    return HERE / "tea_leaf"


def _load(path: pathlib.Path) -> ctypes.CDLL:
    if not path.exists():
        raise RuntimeError(f"{path.name} is not built (run tealeaf-kokkos_b200/build.py); "
                           "there is no CPU fallback")
    return ctypes.CDLL(str(path), mode=ctypes.RTLD_LOCAL)


_LIBS: dict = {}


def load_library(path) -> ctypes.CDLL:
    """Load (once) an ext_* library: the CUDA library or, in tests, an oracle."""
    key = str(pathlib.Path(path).resolve())
    if key not in _LIBS:
        _LIBS[key] = _load(pathlib.Path(key))
    return _LIBS[key]


def cuda_library(dim: int) -> ctypes.CDLL:
    return load_library(lib_path(dim))


# ----------------------------------------------------------------------------- driver


class RunOptions(ctypes.Structure):
    _fields_ = [
        ("dim", ctypes.c_int), ("backend", ctypes.c_char_p), ("use_fused_solve", ctypes.c_int),
        ("summary_every_step", ctypes.c_int), ("end_step_override", ctypes.c_int), ("quiet", ctypes.c_int),
        ("out_path", ctypes.c_char_p), ("eps_override", ctypes.c_double), ("eps_rel_override", ctypes.c_double),
        ("keep_chunk", ctypes.c_int), ("precision", ctypes.c_int), ("ws_net", ctypes.c_int),
        ("ws_mode", ctypes.c_int), ("reserved", ctypes.c_int * 4),
    ]


class StepRecord(ctypes.Structure):
    _fields_ = [
        ("step", ctypes.c_int), ("iterations", ctypes.c_int), ("status", ctypes.c_int),
        ("cheby_steps", ctypes.c_int), ("time", ctypes.c_double), ("dt", ctypes.c_double),
        ("error", ctypes.c_double), ("exact_error", ctypes.c_double), ("eps_used", ctypes.c_double),
        ("solve_seconds", ctypes.c_double), ("vol", ctypes.c_double), ("mass", ctypes.c_double),
        ("ie", ctypes.c_double), ("temp", ctypes.c_double), ("has_summary", ctypes.c_int),
        ("switch_step", ctypes.c_int), ("est_itc", ctypes.c_int), ("warm_start_used", ctypes.c_int),
        ("wall_end", ctypes.c_double), ("h2d_bytes", ctypes.c_longlong), ("d2h_bytes", ctypes.c_longlong),
        ("corrections", ctypes.c_int), ("inner_solver", ctypes.c_int), ("warm_r0_plain", ctypes.c_double),
        ("warm_r0_guess", ctypes.c_double),
    ]


class RunSummary(ctypes.Structure):
    _fields_ = [
        ("steps", ctypes.c_int), ("test_problem", ctypes.c_int), ("kat_available", ctypes.c_int),
        ("kat_passed", ctypes.c_int), ("qa_diff", ctypes.c_double), ("kat_expected", ctypes.c_double),
        ("vol", ctypes.c_double), ("mass", ctypes.c_double), ("ie", ctypes.c_double), ("temp", ctypes.c_double),
        ("wall_seconds", ctypes.c_double), ("solve_seconds", ctypes.c_double), ("total_iterations", ctypes.c_long),
        ("x_cells", ctypes.c_int), ("y_cells", ctypes.c_int), ("z_cells", ctypes.c_int), ("solver", ctypes.c_int),
    ]


def _struct_dict(s) -> dict:
    return {name: getattr(s, name) for name, _ in s._fields_ if name not in ("reserved", "pad")}


def driver() -> ctypes.CDLL:
    lib = load_library(driver_path())
    lib.tea_run_deck.restype = ctypes.c_int
    lib.tea_run_deck.argtypes = [ctypes.c_char_p, ctypes.POINTER(RunOptions), ctypes.POINTER(RunSummary),
                                 ctypes.POINTER(StepRecord), ctypes.c_int]
    lib.tea_driver_last_error.restype = ctypes.c_char_p
    return lib


def run_deck(deck_text: str, dim: int, backend=None, *, fused: bool = False, summary_every_step: bool = False,
             end_step: int = 0, quiet: bool = True, out_path=None, eps: float = 0.0, eps_rel: float = 0.0,
             keep_chunk: bool = False, precision: int = 0, max_records: int = 100000, ws_net: int = 0,
             ws_mode: int = 0, comm=None):
    """Run a tea.in deck through the C++ driver against ``backend`` (default: the CUDA
    library for ``dim``).  Returns ``(summary, records)`` as dicts."""
    backend = str(backend) if backend is not None else str(lib_path(dim))
    if backend == str(lib_path(dim)):
        cuda_library(dim)  # raise early, with a clear message, when it is not built
    opt = RunOptions()
    opt.dim = dim
    opt.backend = backend.encode()
    opt.use_fused_solve = 1 if fused else 0
    opt.summary_every_step = 1 if summary_every_step else 0
    opt.end_step_override = int(end_step)
    opt.quiet = 1 if quiet else 0
    opt.out_path = str(out_path).encode() if out_path else None
    opt.eps_override = float(eps)
    opt.eps_rel_override = float(eps_rel)
    opt.keep_chunk = 1 if keep_chunk else 0
    opt.precision = int(precision)
    opt.ws_net = int(ws_net)
    opt.ws_mode = int(ws_mode)
    summary = RunSummary()
    records = (StepRecord * max_records)()
    lib = driver()
    if comm is None:
        rc = lib.tea_run_deck(deck_text.encode(), ctypes.byref(opt), ctypes.byref(summary), records, max_records)
    else:
        rc = lib.tea_run_deck_comm(deck_text.encode(), ctypes.byref(opt), ctypes.byref(comm), ctypes.byref(summary),
                                   records, max_records)
    if rc != 0:
        raise RuntimeError("tea driver: " + lib.tea_driver_last_error().decode())
    n = min(summary.steps, max_records)
    return _struct_dict(summary), [_struct_dict(records[i]) for i in range(n)]


_ALLREDUCE = ctypes.CFUNCTYPE(None, ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_void_p)
_SENDRECV = ctypes.CFUNCTYPE(None, ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_int,
                             ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_int, ctypes.c_void_p)


class Comm(ctypes.Structure):
    _fields_ = [("rank", ctypes.c_int), ("size", ctypes.c_int), ("allreduce_sum", _ALLREDUCE),
                ("sendrecv", _SENDRECV), ("ctx", ctypes.c_void_p)]


def run_deck_dist(deck_text: str, dim: int, backend=None, *, group=None, device=None, **kw):
    """run_deck over the ranks of a torch.distributed process group: rank r owns the r-th
    slab of the slowest axis; halo faces and global sums go through the group (gloo on the
    host, or NCCL with ``device`` a CUDA device).  Per-call path only."""
    import torch
    import torch.distributed as dist

    def to_dev(t):
        return t.to(device) if device is not None else t

    def allreduce(ptr, n, _ctx):
        a = np.ctypeslib.as_array(ptr, shape=(n,))
        t = to_dev(torch.from_numpy(a.copy()))
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        a[:] = t.cpu().numpy()

    def sendrecv(sp, ns, to, rp, nr, frm, _ctx):
        snd = to_dev(torch.from_numpy(np.ctypeslib.as_array(sp, shape=(ns,)).copy()))
        rcv = to_dev(torch.empty(nr, dtype=torch.float64))
        reqs = [dist.isend(snd, to, group=group), dist.irecv(rcv, frm, group=group)]
        for q in reqs:
            q.wait()
        np.ctypeslib.as_array(rp, shape=(nr,))[:] = rcv.cpu().numpy()

    comm = Comm()
    comm.rank = dist.get_rank(group)
    comm.size = dist.get_world_size(group)
    comm.allreduce_sum = _ALLREDUCE(allreduce)
    comm.sendrecv = _SENDRECV(sendrecv)
    comm.ctx = None
    return run_deck(deck_text, dim, backend, comm=comm, **kw)


# ----------------------------------------------------------------------------- chunks

class SolveParams(ctypes.Structure):
    _fields_ = [
        ("solver", ctypes.c_int), ("coefficient", ctypes.c_int), ("preconditioner", ctypes.c_int),
        ("max_iters", ctypes.c_int), ("ch_cg_presteps", ctypes.c_int), ("ch_cg_errswitch", ctypes.c_int),
        ("ppcg_inner_steps", ctypes.c_int), ("check_result", ctypes.c_int), ("dt", ctypes.c_double),
        ("eps", ctypes.c_double), ("ch_cg_epslim", ctypes.c_double), ("eps_rel", ctypes.c_double),
        ("precision", ctypes.c_int), ("inner_max_iters", ctypes.c_int), ("inner_tol", ctypes.c_double),
        ("inner_solver", ctypes.c_int), ("reserved", ctypes.c_int * 3),
    ]


class SolveResult(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_int), ("status", ctypes.c_int), ("cg_steps", ctypes.c_int),
        ("cheby_steps", ctypes.c_int), ("switch_step", ctypes.c_int), ("est_itc", ctypes.c_int),
        ("error", ctypes.c_double), ("exact_error", ctypes.c_double), ("eps_used", ctypes.c_double),
        ("eigmin", ctypes.c_double), ("eigmax", ctypes.c_double), ("corrections", ctypes.c_int),
        ("warm_start_used", ctypes.c_int), ("warm_r0_plain", ctypes.c_double), ("warm_r0_guess", ctypes.c_double),
        ("inner_solver", ctypes.c_int), ("pad", ctypes.c_int), ("reserved", ctypes.c_double * 4),
    ]


def _i(v):
    return ctypes.byref(ctypes.c_int(int(v)))


def _d(v):
    return ctypes.byref(ctypes.c_double(float(v)))


class ExtChunk:
    """One chunk of an ext_* library, driven call by call.

    ``lib`` is a loaded library exporting the reference ABI plus the inspection entry
    points of include/tea_b200.h.  Fields are exchanged as numpy arrays in the
    reference's flat padded layout, shaped ``(Z, Y, X)`` (``Z == 1`` in 2D)."""

    def __init__(self, lib: ctypes.CDLL, dim: int, nx: int, ny: int, nz: int = 1):
        self.lib, self.dim = lib, dim
        before = self._count()
        if dim == 2:
            lib.ext_init_(_i(nx), _i(ny), _i(0))
        else:
            lib.ext_init_(_i(nx), _i(ny), _i(nz), _i(0))
        self.status()
        self.id = self._find_id(before)
        dims = (ctypes.c_int * 3)()
        if lib.tea_chunk_dims_(ctypes.byref(ctypes.c_int(self.id)), dims) != 0:
            raise RuntimeError("chunk not created")
        self.X, self.Y, self.Z = dims[0], dims[1], dims[2]

    def _count(self):
        dims = (ctypes.c_int * 3)()
        n = 0
        while self.lib.tea_chunk_dims_(ctypes.byref(ctypes.c_int(n + 1)), dims) == 0:
            n += 1
        return n

    def _find_id(self, before):
        after = self._count()
        if after != before + 1:
            raise RuntimeError(f"ext_init_ did not add a chunk ({before} -> {after})")
        return after

    @property
    def cid(self):
        return ctypes.byref(ctypes.c_int(self.id))

    def status(self):
        if hasattr(self.lib, "ext_get_status_"):
            st = ctypes.c_int(0)
            self.lib.ext_get_status_(ctypes.byref(st))
            if st.value not in (0, 7):
                msg = ""
                if hasattr(self.lib, "tea_last_error"):
                    self.lib.tea_last_error.restype = ctypes.c_char_p
                    msg = self.lib.tea_last_error().decode()
                raise RuntimeError(f"ext library status {st.value}: {msg}")

    def read(self, field: str) -> np.ndarray:
        out = np.empty((self.Z, self.Y, self.X), dtype=np.float64)
        rc = self.lib.tea_read_field_(self.cid, _i(FIELD_IDS[field]), out.ctypes.data_as(ctypes.c_void_p))
        if rc != 0:
            raise RuntimeError(f"read of {field} failed")
        return out

    def write(self, field: str, arr: np.ndarray) -> None:
        a = np.ascontiguousarray(arr, dtype=np.float64).reshape(self.Z, self.Y, self.X)
        rc = self.lib.tea_write_field_(self.cid, _i(FIELD_IDS[field]), a.ctypes.data_as(ctypes.c_void_p))
        if rc != 0:
            raise RuntimeError(f"write of {field} failed")

    # thin wrappers over the reference entry points ------------------------------------
    def initialise(self, xmin, ymin, dx, dy, zmin=0.0, dz=1.0):
        if self.dim == 2:
            self.lib.ext_initialise_chunk_(self.cid, _d(xmin), _d(ymin), _d(dx), _d(dy))
        else:
            self.lib.ext_initialise_chunk_(self.cid, _d(xmin), _d(ymin), _d(zmin), _d(dx), _d(dy), _d(dz))
        self.status()

    def reduce(self, name, *args):
        out = ctypes.c_double(0.0)
        getattr(self.lib, name)(self.cid, *args, ctypes.byref(out))
        self.status()
        return out.value

    def norm2(self, use_r):
        """ext_calculate_2norm_: the norm comes back through the second argument, ahead of the flag."""
        out = ctypes.c_double(0.0)
        self.lib.ext_calculate_2norm_(self.cid, ctypes.byref(out), ctypes.byref(ctypes.c_int(1 if use_r else 0)))
        self.status()
        return out.value

    def call(self, name, *args):
        getattr(self.lib, name)(self.cid, *args)
        self.status()

    def field_summary(self):
        v = [ctypes.c_double(0.0) for _ in range(4)]
        self.lib.ext_field_summary_kernel_(self.cid, *[ctypes.byref(x) for x in v])
        self.status()
        return tuple(x.value for x in v)

    def update_halo(self, fields, depth, neighbours=None):
        nb = (ctypes.c_int * 6)(*(neighbours or [-1] * 6))
        fl = (ctypes.c_int * 6)(*[1 if (k + 1) in fields else 0 for k in range(6)])
        self.lib.ext_update_halo_kernel_(self.cid, nb, fl, _i(depth))
        self.status()

    def solve(self, params: SolveParams) -> dict:
        res = SolveResult()
        self.lib.ext_tea_leaf_solve_(self.cid, ctypes.byref(params), ctypes.byref(res))
        self.status()
        return _struct_dict(res)


# ----------------------------------------------------------------------------- decks

WS_RECORD, WS_ATTACH = 1, 2  # run_deck ws_mode values


class WarmStart:
    """A learned warm-start network of the 2D or the 3D CUDA library (tea_ws_* entry
    points): 3x3 convolutions over images in 2D, 3x3x3 convolutions over volumes in 3D."""

    def __init__(self, levels: int = 3, base: int = 32, seed: int = 0, dim: int = 2, max_channels: int = 0):
        self.lib = cuda_library(dim)
        self.dim = dim
        nid = ctypes.c_int(0)
        self._check(self.lib.tea_ws_create_capped_(_i(levels), _i(base), _i(max_channels), _i(seed),
                                                   ctypes.byref(nid)), "create")
        self.id = nid.value
        self.levels, self.base, self.max_channels = levels, base, max_channels

    def _check(self, rc, what):
        if rc != 0:
            self.lib.tea_last_error.restype = ctypes.c_char_p
            raise RuntimeError(f"tea_ws_{what}_: status {rc}: {self.lib.tea_last_error().decode()}")

    def close(self):
        if self.id:
            self.lib.tea_ws_destroy_(_i(self.id))
            self.id = 0

    def param_count(self) -> int:
        n = ctypes.c_longlong(0)
        self._check(self.lib.tea_ws_param_count_(_i(self.id), ctypes.byref(n)), "param_count")
        return n.value

    def get_params(self) -> np.ndarray:
        out = np.zeros(self.param_count(), dtype=np.float32)
        self._check(self.lib.tea_ws_get_params_(_i(self.id), out.ctypes.data_as(ctypes.c_void_p)), "get_params")
        return out

    def set_params(self, flat) -> None:
        arr = np.ascontiguousarray(flat, dtype=np.float32)
        self._check(self.lib.tea_ws_set_params_(_i(self.id), arr.ctypes.data_as(ctypes.c_void_p)), "set_params")

    def set_reference_conv(self, on: bool) -> None:
        self._check(self.lib.tea_ws_set_conv_(_i(self.id), _i(1 if on else 0)), "set_conv")

    def set_conv_mode(self, mode: int) -> None:
        """0: tensor cores (TMA-fed where the width is a multiple of 128), 1: CUDA cores,
        2: tensor cores without TMA."""
        self._check(self.lib.tea_ws_set_conv_(_i(self.id), _i(mode)), "set_conv")

    def eval(self, x, target=None, kxy=None):
        """x [n][H][W][4] (2D) or [n][D][H][W][5] (3D) float32 -> (y [n][(D)][H][W], loss,
        flat gradients or None); with kxy ([n][(D)][H][W][dim] face coefficients) the loss is
        the residual loss of training."""
        x = np.ascontiguousarray(x, dtype=np.float32)
        if self.dim == 3:
            n, D, H, W, _ = x.shape
        else:
            (n, H, W, _), D = x.shape, 1
        y = np.zeros(x.shape[:-1], dtype=np.float32)
        loss = ctypes.c_double(0.0)
        grads = np.zeros(self.param_count(), dtype=np.float32) if target is not None else None
        t = np.ascontiguousarray(target, dtype=np.float32) if target is not None else None
        k = np.ascontiguousarray(kxy, dtype=np.float32) if kxy is not None else None
        P = lambda a: a.ctypes.data_as(ctypes.c_void_p) if a is not None else None
        self._check(self.lib.tea_ws_eval_volume_(_i(self.id), P(x), P(t), P(k), _i(n), _i(D), _i(H), _i(W), P(y),
                                                 ctypes.byref(loss), P(grads)), "eval_volume")
        return y, loss.value, grads

    def pairs(self) -> int:
        n = ctypes.c_int(0)
        self._check(self.lib.tea_ws_pairs_(_i(self.id), ctypes.byref(n)), "pairs")
        return n.value

    def train(self, steps: int, batch: int, crop: int, lr: float = 1e-3, seed: int = 0):
        """Returns (first-step loss, last-step loss, device ms per step)."""
        lf, ll, ms = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.tea_ws_train_(_i(self.id), _i(steps), _i(batch), _i(crop), _d(lr), _i(seed),
                                           ctypes.byref(lf), ctypes.byref(ll), ctypes.byref(ms)), "train")
        return lf.value, ll.value, ms.value


@dataclass
class DeckSpec:
    dim: int = 2
    cells: int = 512
    states: int = 6
    seed: int = 0
    solver: str = "cg"
    end_step: int = 10
    dt: float = 0.004
    eps: float = 1e-15
    eps_rel: float = 0.0
    max_iters: int = 10000
    presteps: int = 30
    inner_steps: int = 10
    domain: float = 10.0
    inverse_density: bool = True
    preconditioner: bool = False
    check_result: bool = True
    test_problem: int = 0
    summary_frequency: int = 10


def seeded_deck(spec: DeckSpec) -> str:
    """A tea.in deck of the seeded synthetic layouts: state 1 ambient (density 100,
    energy 1e-4); states 2..N rectangles/cuboids or circles/spheres with probability
    1/2 each, density log-uniform in [0.1, 100], energy uniform in [1, 25], positions
    uniform in the domain, extents uniform in (0, domain/2], radii in (0, domain/4];
    the last state takes priority.  numpy's PCG64 with ``spec.seed``."""
    rng = np.random.Generator(np.random.PCG64(spec.seed))
    L = spec.domain
    lines = ["*tea", "state 1 density=100.0 energy=0.0001"]
    for s in range(2, spec.states + 1):
        den = float(10.0 ** rng.uniform(-1.0, 2.0))
        en = float(rng.uniform(1.0, 25.0))
        if rng.uniform() < 0.5:
            geo = "rectangle" if spec.dim == 2 else "cuboid"
            x0, y0, z0 = (float(v) for v in rng.uniform(0, L, 3))
            wx, wy, wz = (float(L / 2 - v) for v in rng.uniform(0, L / 2, 3))  # (0, L/2]
            box = f"xmin={x0!r} xmax={x0 + wx!r} ymin={y0!r} ymax={y0 + wy!r}"
            if spec.dim == 3:
                box += f" zmin={z0!r} zmax={z0 + wz!r}"
            lines.append(f"state {s} density={den!r} energy={en!r} geometry={geo} {box}")
        else:
            x0, y0, z0 = (float(v) for v in rng.uniform(0, L, 3))
            rad = float(L / 4 - rng.uniform(0, L / 4))
            ctr = f"xmin={x0!r} ymin={y0!r}" + (f" zmin={z0!r}" if spec.dim == 3 else "")
            lines.append(f"state {s} density={den!r} energy={en!r} geometry=circle {ctr} radius={rad!r}")
    lines += [f"x_cells={spec.cells}", f"y_cells={spec.cells}"]
    if spec.dim == 3:
        lines.append(f"z_cells={spec.cells}")
    lines += ["xmin=0.0", "ymin=0.0", f"xmax={L!r}", f"ymax={L!r}"]
    if spec.dim == 3:
        lines += ["zmin=0.0", f"zmax={L!r}"]
    lines += [f"initial_timestep={spec.dt!r}", f"end_step={spec.end_step}", f"tl_max_iters={spec.max_iters}",
              f"summary_frequency={spec.summary_frequency}",
              SOLVER_KEYWORDS[SOLVERS[spec.solver]], f"tl_eps={spec.eps!r}",
              f"tl_ch_cg_presteps={spec.presteps}", f"tl_ppcg_inner_steps={spec.inner_steps}"]
    if spec.eps_rel > 0:
        lines.append(f"tl_eps_rel={spec.eps_rel!r}")
    if spec.inverse_density:
        lines.append("tl_coefficient_inverrse_density")
    if spec.preconditioner:
        lines.append("tl_preconditioner_on")
    if spec.check_result:
        lines.append("tl_check_result")
    if spec.test_problem:
        lines.append(f"test_problem {spec.test_problem}")
    lines.append("*endtea")
    return "\n".join(lines) + "\n"


def rel_diff(a: float, b: float) -> float:
    if a == b:
        return 0.0
    if math.isnan(a) or math.isnan(b):
        return math.inf
    return abs(a - b) / max(abs(a), abs(b), 1e-300)


def build(verbose: bool = False, force: bool = False) -> None:
    """Compile the CUDA libraries and the driver in-tree (see build.py)."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("_tea_b200_build", HERE / "build.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    mod.build(verbose=verbose, force=force)


__all__ = [
    "FIELD_IDS", "SOLVERS", "PRECISION_FP64", "PRECISION_FP32_REFINED", "lib_path", "driver_path", "tea_leaf_exe", "load_library", "cuda_library",
    "run_deck", "ExtChunk", "SolveParams", "SolveResult", "DeckSpec", "seeded_deck", "rel_diff", "build",
]

if os.environ.get("TEA_B200_BUILD_ON_IMPORT"):
    build()
