"""The solve split into slabs over several ranks (the reference's MPI layer: tea_decompose,
tea_exchange, tea_allsum) -- here two and three gloo ranks on the host, each running the
C++ driver against the oracle port, against the single-rank run.

Every global scalar becomes a sum of per-rank partial sums, which may differ from the
single-chunk sum in the last bit, so the bar is the one used against the reference's own
plain sums: iteration counts within 1 and field summaries within 1e-10 relative.

The exchange packs faces with tea_pack_face_: the reference's 2D bottom/top packer
(tealeaf_2d/ext_pack_kernel.hpp:17-44, kept as ext_pack_message_) starts at padded column 0,
which leaves the last two inner columns of every exchanged halo row stale.
"""
import ctypes
import json
import os
import socket

import numpy as np
import pytest

from conftest import PORT, SUM_COMPENSATED, port_lib, rel, tea

CASES = [(2, "cg"), (2, "chebyshev"), (2, "ppcg"), (2, "jacobi"), (3, "cg"), (3, "ppcg")]


def _deck(dim, solver):
    spec = tea.DeckSpec(dim=dim, cells=40 if dim == 2 else 14, states=6, seed=77, solver=solver, end_step=3,
                        eps=1e-15, eps_rel=1e-10, max_iters=5000, summary_frequency=1, check_result=True)
    return tea.seeded_deck(spec)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, size, port, out_dir, on_gpu=False):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=size)
    try:
        res = {}
        for dim, solver in CASES:
            backend = None if on_gpu else port_lib(dim, SUM_COMPENSATED)  # None: the CUDA library
            _, recs = tea.run_deck_dist(_deck(dim, solver), dim, backend, summary_every_step=True)
            res[f"{dim}_{solver}"] = recs
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump(res, f)
    finally:
        dist.destroy_process_group()


def _run_ranks(tmp_path, ranks, on_gpu):
    import torch.multiprocessing as mp

    mp.start_processes(_rank, args=(ranks, _free_port(), str(tmp_path), on_gpu), nprocs=ranks, join=True,
                       start_method="spawn")
    return [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in range(ranks)]


@pytest.mark.parametrize("ranks", [2, 3])
def test_slabs_match_one_rank(tmp_path, ranks):
    """Three ranks split 40 rows as 14/13/13 and 14 planes as 5/5/4 (tea_decompose's remainder
    rule), so the ragged split is covered too."""
    _check_against_one_rank(_run_ranks(tmp_path, ranks, False), ranks)


@pytest.mark.gpu
def test_slabs_on_the_cuda_library_match_one_rank(tmp_path):
    """The same two-rank split with every rank's chunk in the CUDA library.  Both ranks share
    the one GPU; they meet only in host-side gloo calls between kernel launches (no kernel
    waits on another rank)."""
    _check_against_one_rank(_run_ranks(tmp_path, 2, True), 2)


def _check_against_one_rank(got, ranks):
    for dim, solver in CASES:
        _, ref = tea.run_deck(_deck(dim, solver), dim, port_lib(dim, SUM_COMPENSATED), summary_every_step=True)
        for r in range(ranks):
            recs = got[r][f"{dim}_{solver}"]
            assert len(recs) == len(ref)
            for a, b in zip(recs, ref):
                assert abs(a["iterations"] - b["iterations"]) <= 1, (dim, solver, a["step"])
                for k in ("vol", "mass", "ie", "temp"):
                    assert rel(a[k], b[k]) <= 1e-10, (dim, solver, a["step"], k, a[k], b[k])


def test_whole_solve_path_refuses_several_ranks():
    class Fake:  # a two-rank communicator that must not be called
        pass

    comm = tea.Comm()
    comm.rank, comm.size = 0, 2
    comm.allreduce_sum = tea._ALLREDUCE(lambda *a: None)
    comm.sendrecv = tea._SENDRECV(lambda *a: None)
    with pytest.raises(RuntimeError, match="one chunk"):
        tea.run_deck(_deck(2, "cg"), 2, port_lib(2, SUM_COMPENSATED), fused=True, comm=comm)


def _i(v):
    return ctypes.byref(ctypes.c_int(v))


@pytest.mark.parametrize("face", [3, 4])
def test_face_packers_2d(face):
    """Bottom (3) and top (4) faces, depth 2: tea_pack_face_ sends the inner columns 2..nx+1 of
    the two rows next to the face; ext_pack_message_ sends columns 0..nx-1 of the same rows,
    as the reference does."""
    port_lib(2, SUM_COMPENSATED)
    lib = tea.load_library(PORT[2])
    nx, ny, depth = 9, 7, 2
    ch = tea.ExtChunk(lib, 2, nx, ny, 1)
    try:
        X, Y = ch.X, ch.Y
        dens = np.arange(X * Y, dtype=np.float64).reshape(1, Y, X)
        ch.write("density", dens)
        rows = [2, 3] if face == 3 else [Y - 4, Y - 3]
        fields = (ctypes.c_int * 6)(1, 0, 0, 0, 0, 0)
        offsets = (ctypes.c_int * 6)(0, 0, 0, 0, 0, 0)
        got = {}
        for name in ("tea_pack_face_", "ext_pack_message_"):
            buf = np.zeros(nx * depth)
            ch.call(name, fields, offsets, _i(depth), _i(face), buf.ctypes.data_as(ctypes.c_void_p), _i(1))
            got[name] = buf.reshape(depth, nx)
        assert np.array_equal(got["tea_pack_face_"], dens[0, rows, 2:nx + 2])
        assert np.array_equal(got["ext_pack_message_"], dens[0, rows, 0:nx])
        # Unpacking puts the exact packer's rows into the halo rows on the inner columns only.
        src = -1.0 - np.arange(nx * depth, dtype=np.float64)
        ch.call("tea_pack_face_", fields, offsets, _i(depth), _i(face), src.ctypes.data_as(ctypes.c_void_p), _i(0))
        halo = [0, 1] if face == 3 else [Y - 2, Y - 1]
        after = ch.read("density")
        assert np.array_equal(after[0, halo, 2:nx + 2], src.reshape(depth, nx))
        untouched = np.ones_like(dens, dtype=bool)
        untouched[0, halo, 2:nx + 2] = False
        assert np.array_equal(after[untouched], dens[untouched])
    finally:
        lib.ext_finalise_()
